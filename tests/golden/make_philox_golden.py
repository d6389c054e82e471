"""Generate tests/golden/philox_curand.npz from cuRAND's host Philox4_32_10.

cuRAND's host generator is an independent implementation of Philox4x32-10
(Salmon et al., SC11): with seed s its i-th 128-bit output block is Philox at
key (s lo, s hi) and counter (i / 65536, 0, i % 65536, 0) -- the generator
spreads its output over 65536 subsequences (counter word 2) and advances the
position inside each subsequence in counter word 0.  That layout was found by
matching the generator's output against this repository's oracle; the test
then checks all listed blocks, so a wrong layout or a wrong Philox fails.
Run once on any machine with libcurand (no GPU needed); the .npz is
committed so the test never needs cuRAND.
"""
import ctypes
import os

import numpy as np

CURAND_RNG_PSEUDO_PHILOX4_32_10 = 161


def curand_blocks(seed, offset_blocks, n_blocks):
    lib = ctypes.CDLL(os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "lib64", "libcurand.so"))
    gen = ctypes.c_void_p()
    assert lib.curandCreateGeneratorHost(ctypes.byref(gen), CURAND_RNG_PSEUDO_PHILOX4_32_10) == 0
    assert lib.curandSetPseudoRandomGeneratorSeed(gen, ctypes.c_ulonglong(seed)) == 0
    assert lib.curandSetGeneratorOffset(gen, ctypes.c_ulonglong(offset_blocks * 4)) == 0
    out = np.zeros(4 * n_blocks, dtype=np.uint32)
    assert lib.curandGenerate(gen, out.ctypes.data_as(ctypes.c_void_p), ctypes.c_size_t(out.size)) == 0
    lib.curandDestroyGenerator(gen)
    return out.reshape(n_blocks, 4)


def main():
    cases = []
    # (seed, first block index, number of blocks)
    for seed, off, n in [(0, 0, 8), (0xDEADBEEF12345678, 0, 8), (42, (1 << 16) - 3, 6),
                         (42, (1 << 40) + 17, 4), (0xFFFFFFFFFFFFFFFF, 123456789, 4)]:
        blocks = curand_blocks(seed, off, n)
        for i in range(n):
            idx = off + i
            ctr = [(idx >> 16) & 0xFFFFFFFF, 0, idx & 0xFFFF, 0]
            key = [seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF]
            cases.append(ctr + key + list(blocks[i]))
    arr = np.array(cases, dtype=np.uint32)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "philox_curand.npz")
    np.savez(out, cases=arr)
    print(f"wrote {arr.shape[0]} Philox blocks to {out}")


if __name__ == "__main__":
    main()
