"""The reference's own CPU path built as a test oracle (see run.py)."""
