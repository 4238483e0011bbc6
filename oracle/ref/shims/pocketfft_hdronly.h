// Stand-in for the one PocketFFT entry point the reference's serial FFT grid calls
// (pocketfft::c2c, used by src/layer_3_representation/basis/planewave/internal/fft/
// fft_grid_serial_pocket.hpp:132-143), for building the reference's CPU path as a
// test oracle.  PocketFFT itself (mreineck/pocketfft, commit c90e55b3, the revision the
// reference's CMakeLists.txt:295-297 fetches) is not in this environment, so the
// arithmetic here is our own:
//
//   * a Stockham autosort mixed-radix FFT, decimation in frequency, natural order out,
//     with radix 4, 2, 3 and 5 butterflies and any other prime factor by its direct DFT;
//   * twiddles exp(-+2 pi i j / n) computed in long double and rounded once, laid out per
//     stage so the butterflies read them in order;
//   * lines are transformed in panels of V lines held as a [n][V] buffer, so every
//     butterfly runs over V independent lines with unit stride (the compiler vectorises
//     the V loop); along a strided axis a panel is V neighbouring lines, along the
//     contiguous axis it is V consecutive lines gathered by a small transpose.
//
// Contract kept from PocketFFT: forward = exp(-i 2 pi jk/n), unnormalised; the result
// is multiplied by `fct`; input and output may alias; strides are in bytes; the
// transform is split over `nthreads` OpenMP threads.
#pragma once

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstddef>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

namespace pocketfft {

using shape_t = std::vector<std::size_t>;
using stride_t = std::vector<std::ptrdiff_t>;

namespace shim {

using cd = std::complex<double>;

struct Stage {
    std::size_t p, m, s;        // radix, remaining length after it, product of radices before
    std::vector<cd> tw;         // tw[j*(p-1) + (k-1)] = W_{m p}^{j k}, j < m, 1 <= k < p
    std::vector<cd> wp;         // W_p^{t}, t < p (generic radix only)
};

struct Plan {
    std::size_t n = 0;
    std::vector<Stage> fwd, bwd;
};

inline cd unit(long double turns) {
    const long double two_pi = 6.283185307179586476925286766559005768L;
    long double a = two_pi * turns;
    return cd(static_cast<double>(std::cos(a)), static_cast<double>(std::sin(a)));
}

inline std::shared_ptr<const Plan> plan_for(std::size_t n) {
    static std::mutex mu;
    static std::map<std::size_t, std::shared_ptr<const Plan>> cache;
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(n);
    if (it != cache.end()) return it->second;
    auto plan = std::make_shared<Plan>();
    plan->n = n;
    std::vector<std::size_t> radices;
    std::size_t r = n;
    while (r % 4 == 0) { radices.push_back(4); r /= 4; }
    while (r % 2 == 0) { radices.push_back(2); r /= 2; }
    for (std::size_t f : {3u, 5u}) while (r % f == 0) { radices.push_back(f); r /= f; }
    for (std::size_t f = 7; r > 1; f += 2) while (r % f == 0) { radices.push_back(f); r /= f; }
    for (int dir = 0; dir < 2; ++dir) {
        const long double sign = dir == 0 ? -1.0L : 1.0L;
        std::size_t m = n, s = 1;
        auto& stages = dir == 0 ? plan->fwd : plan->bwd;
        for (std::size_t p : radices) {
            m /= p;
            Stage st{p, m, s, {}, {}};
            st.tw.resize(m * (p - 1));
            for (std::size_t j = 0; j < m; ++j)
                for (std::size_t k = 1; k < p; ++k)
                    st.tw[j * (p - 1) + (k - 1)] =
                        unit(sign * static_cast<long double>(j * k) / static_cast<long double>(m * p));
            st.wp.resize(p);
            for (std::size_t t = 0; t < p; ++t)
                st.wp[t] = unit(sign * static_cast<long double>(t) / static_cast<long double>(p));
            stages.push_back(std::move(st));
            s *= p;
        }
    }
    cache.emplace(n, plan);
    return plan;
}

// One Stockham stage on V-wide rows:
//   y[q + s (p j + k)] = W_{mp}^{jk} sum_r x[q + s (j + r m)] W_p^{rk}
// with row index t holding V values at buf[t*V .. t*V+V).
inline void run_stage(const Stage& st, bool forward, std::size_t V, const cd* __restrict x,
                      cd* __restrict y) {
    const std::size_t p = st.p, m = st.m, s = st.s;
    const std::size_t xr = s * m * V;   // row distance between r and r+1
    const std::size_t yk = s * V;       // row distance between k and k+1
    for (std::size_t j = 0; j < m; ++j) {
        const cd* tw = st.tw.data() + j * (p - 1);
        for (std::size_t q = 0; q < s; ++q) {
            const cd* xi = x + (q + s * j) * V;
            cd* yo = y + (q + s * p * j) * V;
            if (p == 4) {
                const cd w1 = tw[0], w2 = tw[1], w3 = tw[2];
                const double sg = forward ? -1.0 : 1.0;  // multiply by -i (fwd) or +i (bwd)
                for (std::size_t v = 0; v < V; ++v) {
                    const cd a0 = xi[v], a1 = xi[xr + v], a2 = xi[2 * xr + v], a3 = xi[3 * xr + v];
                    const cd t0 = a0 + a2, t1 = a0 - a2, t2 = a1 + a3, d = a1 - a3;
                    const cd t3(-sg * d.imag(), sg * d.real());
                    yo[v] = t0 + t2;
                    yo[yk + v] = (t1 + t3) * w1;
                    yo[2 * yk + v] = (t0 - t2) * w2;
                    yo[3 * yk + v] = (t1 - t3) * w3;
                }
            } else if (p == 2) {
                const cd w1 = tw[0];
                for (std::size_t v = 0; v < V; ++v) {
                    const cd a0 = xi[v], a1 = xi[xr + v];
                    yo[v] = a0 + a1;
                    yo[yk + v] = (a0 - a1) * w1;
                }
            } else if (p == 3) {
                const cd w1 = tw[0], w2 = tw[1];
                const double c = -0.5, sn = (forward ? -1.0 : 1.0) * 0.86602540378443864676;
                for (std::size_t v = 0; v < V; ++v) {
                    const cd a0 = xi[v], a1 = xi[xr + v], a2 = xi[2 * xr + v];
                    const cd sum = a1 + a2, dif = a1 - a2;
                    const cd mid = a0 + c * sum;
                    const cd rot(-sn * dif.imag(), sn * dif.real());
                    yo[v] = a0 + sum;
                    yo[yk + v] = (mid + rot) * w1;
                    yo[2 * yk + v] = (mid - rot) * w2;
                }
            } else if (p == 5) {
                const cd w1 = tw[0], w2 = tw[1], w3 = tw[2], w4 = tw[3];
                const double c1 = st.wp[1].real(), c2 = st.wp[2].real();
                const double s1 = st.wp[1].imag(), s2 = st.wp[2].imag();
                for (std::size_t v = 0; v < V; ++v) {
                    const cd a0 = xi[v], a1 = xi[xr + v], a2 = xi[2 * xr + v], a3 = xi[3 * xr + v],
                             a4 = xi[4 * xr + v];
                    const cd b1 = a1 + a4, b4 = a1 - a4, b2 = a2 + a3, b3 = a2 - a3;
                    const cd m1 = a0 + c1 * b1 + c2 * b2, m2 = a0 + c2 * b1 + c1 * b2;
                    // i*(s1 b4 + s2 b3) and i*(s2 b4 - s1 b3)
                    const cd u1 = s1 * b4 + s2 * b3, u2 = s2 * b4 - s1 * b3;
                    const cd r1(-u1.imag(), u1.real()), r2(-u2.imag(), u2.real());
                    yo[v] = a0 + b1 + b2;
                    yo[yk + v] = (m1 + r1) * w1;
                    yo[2 * yk + v] = (m2 + r2) * w2;
                    yo[3 * yk + v] = (m2 - r2) * w3;
                    yo[4 * yk + v] = (m1 - r1) * w4;
                }
            } else {
                for (std::size_t v = 0; v < V; ++v) {
                    for (std::size_t k = 0; k < p; ++k) {
                        cd acc = xi[v];
                        for (std::size_t rr = 1; rr < p; ++rr) acc += xi[rr * xr + v] * st.wp[(rr * k) % p];
                        yo[k * yk + v] = k == 0 ? acc : acc * tw[k - 1];
                    }
                }
            }
        }
    }
}

// Transform the n rows of buf (each V wide) in place; work has room for n*V.
inline void fft_panel(const Plan& plan, bool forward, std::size_t V, cd* buf, cd* work) {
    const auto& stages = forward ? plan.fwd : plan.bwd;
    cd* x = buf;
    cd* y = work;
    for (const Stage& st : stages) {
        run_stage(st, forward, V, x, y);
        std::swap(x, y);
    }
    if (x != buf) std::memcpy(buf, x, plan.n * V * sizeof(cd));
}

}  // namespace shim

template <typename T>
void c2c(const shape_t& shape, const stride_t& stride_in, const stride_t& stride_out,
         const shape_t& axes, bool forward, const std::complex<T>* data_in,
         std::complex<T>* data_out, T fct, std::size_t nthreads = 1) {
    static_assert(sizeof(T) == sizeof(double), "the oracle's FFT stand-in is double only");
    using shim::cd;
    const std::size_t nd = shape.size();
    std::size_t total = 1;
    for (auto e : shape) total *= e;
    if (total == 0) return;
    const int threads = static_cast<int>(std::max<std::size_t>(nthreads, 1));

    // Work on a dense row-major copy unless the output already is one.
    bool out_dense = true;
    {
        std::ptrdiff_t expect = static_cast<std::ptrdiff_t>(sizeof(cd));
        for (std::size_t d = nd; d-- > 0;) {
            if (stride_out[d] != expect) out_dense = false;
            expect *= static_cast<std::ptrdiff_t>(shape[d]);
        }
    }
    std::vector<cd> scratch;
    cd* dense = reinterpret_cast<cd*>(data_out);
    if (!out_dense) {
        scratch.resize(total);
        dense = scratch.data();
    }
    {
        std::vector<std::size_t> idx(nd, 0);
        bool in_dense = true;
        std::ptrdiff_t expect = static_cast<std::ptrdiff_t>(sizeof(cd));
        for (std::size_t d = nd; d-- > 0;) {
            if (stride_in[d] != expect) in_dense = false;
            expect *= static_cast<std::ptrdiff_t>(shape[d]);
        }
        if (in_dense) {
            if (reinterpret_cast<const void*>(data_in) != reinterpret_cast<void*>(dense))
                std::memmove(dense, data_in, total * sizeof(cd));
        } else {
            for (std::size_t e = 0; e < total; ++e) {
                std::size_t rem = e;
                std::ptrdiff_t off = 0;
                for (std::size_t d = nd; d-- > 0;) {
                    off += static_cast<std::ptrdiff_t>(rem % shape[d]) * stride_in[d];
                    rem /= shape[d];
                }
                dense[e] = *reinterpret_cast<const cd*>(reinterpret_cast<const char*>(data_in) + off);
            }
        }
    }

    constexpr std::size_t kPanel = 16;  // lines per panel
    for (std::size_t axis : axes) {
        const std::size_t n = shape[axis];
        if (n <= 1) continue;
        std::size_t inner = 1, outer = 1;
        for (std::size_t d = axis + 1; d < nd; ++d) inner *= shape[d];
        for (std::size_t d = 0; d < axis; ++d) outer *= shape[d];
        auto plan = shim::plan_for(n);
        // panels: along a strided axis, kPanel neighbouring inner positions of one outer
        // block; along the contiguous axis, kPanel consecutive lines
        const std::size_t per_outer = inner > 1 ? (inner + kPanel - 1) / kPanel : 1;
        const std::size_t npanels = inner > 1 ? outer * per_outer : (outer + kPanel - 1) / kPanel;
#pragma omp parallel num_threads(threads) if (threads > 1)
        {
            std::vector<cd> buf(n * kPanel), work(n * kPanel);
#pragma omp for schedule(static)
            for (long long pi = 0; pi < static_cast<long long>(npanels); ++pi) {
                if (inner > 1) {
                    const std::size_t o = static_cast<std::size_t>(pi) / per_outer;
                    const std::size_t i0 = (static_cast<std::size_t>(pi) % per_outer) * kPanel;
                    const std::size_t V = std::min(kPanel, inner - i0);
                    cd* base = dense + o * n * inner + i0;
                    for (std::size_t t = 0; t < n; ++t) std::memcpy(&buf[t * V], base + t * inner, V * sizeof(cd));
                    shim::fft_panel(*plan, forward, V, buf.data(), work.data());
                    for (std::size_t t = 0; t < n; ++t) std::memcpy(base + t * inner, &buf[t * V], V * sizeof(cd));
                } else {
                    const std::size_t l0 = static_cast<std::size_t>(pi) * kPanel;
                    const std::size_t V = std::min(kPanel, outer - l0);
                    cd* base = dense + l0 * n;
                    for (std::size_t v = 0; v < V; ++v)
                        for (std::size_t t = 0; t < n; ++t) buf[t * V + v] = base[v * n + t];
                    shim::fft_panel(*plan, forward, V, buf.data(), work.data());
                    for (std::size_t v = 0; v < V; ++v)
                        for (std::size_t t = 0; t < n; ++t) base[v * n + t] = buf[t * V + v];
                }
            }
        }
    }

    const double scale = static_cast<double>(fct);
    if (out_dense) {
        if (scale != 1.0)
            for (std::size_t e = 0; e < total; ++e) dense[e] *= scale;
    } else {
        for (std::size_t e = 0; e < total; ++e) {
            std::size_t rem = e;
            std::ptrdiff_t off = 0;
            for (std::size_t d = nd; d-- > 0;) {
                off += static_cast<std::ptrdiff_t>(rem % shape[d]) * stride_out[d];
                rem /= shape[d];
            }
            *reinterpret_cast<cd*>(reinterpret_cast<char*>(data_out) + off) = dense[e] * scale;
        }
    }
}

}  // namespace pocketfft
