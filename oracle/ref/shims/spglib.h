/* Stand-in for spglib's C header, for building the reference's CPU path as a
 * test oracle.  The oracle harness passes explicit k-point lists and never asks
 * for symmetry, so every query answers "no dataset": callers fall back to the
 * identity (one operation, no k-point reduction). */
#pragma once
#include <stdlib.h>

typedef struct {
    int spacegroup_number;
    char international_symbol[11];
    int n_operations;
    int (*rotations)[3][3];
    double (*translations)[3];
} SpglibDataset;

static inline SpglibDataset* spg_get_dataset(const double lattice[3][3], const double position[][3],
                                             const int types[], int num_atom, double symprec) {
    (void)lattice; (void)position; (void)types; (void)num_atom; (void)symprec;
    return NULL;
}

static inline void spg_free_dataset(SpglibDataset* dataset) { (void)dataset; }

static inline int spg_get_ir_reciprocal_mesh(int grid_address[][3], int ir_mapping_table[],
                                             const int mesh[3], const int is_shift[3],
                                             int is_time_reversal, const double lattice[3][3],
                                             const double position[][3], const int types[],
                                             int num_atom, double symprec) {
    (void)is_shift; (void)is_time_reversal; (void)lattice; (void)position; (void)types;
    (void)num_atom; (void)symprec;
    int n = mesh[0] * mesh[1] * mesh[2];
    for (int i = 0; i < n; ++i) {
        ir_mapping_table[i] = i;
        grid_address[i][0] = i % mesh[0];
        grid_address[i][1] = (i / mesh[0]) % mesh[1];
        grid_address[i][2] = i / (mesh[0] * mesh[1]);
    }
    return n;
}
