"""The reference tests' xorshift32 generator (src/fluid_core.rs:11234-11240),
returning float32 values exactly as the Rust closure does."""
import numpy as np


class XorShift:
    def __init__(self, seed):
        self.s = seed & 0xFFFFFFFF

    def next(self):
        s = self.s
        s ^= (s << 13) & 0xFFFFFFFF
        s ^= s >> 17
        s ^= (s << 5) & 0xFFFFFFFF
        self.s = s
        return np.float32(s >> 8) / np.float32(1 << 24)
