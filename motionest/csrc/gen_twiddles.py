"""Generate dft_consts.cuh: DFT twiddle constants as literals.

  python motionest/csrc/gen_twiddles.py   (run by motionest/build.py when the header is stale)

Emits, for every line length the compile-time FFT kernels support, a global device table
tw<N>[m] = exp(-2 pi i m / N) (m < N), initialised in the module image (no set-up kernel), the
same values in the order of the second FFT stage (twp<N>), and
for every small radix R the constants cos(2 pi m / R), sin(2 pi m / R) used by the register
DFTs.  The values are plain float64 evaluations of cos/sin rounded to float32.
"""
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
OUT = HERE / "dft_consts.cuh"

# Line lengths with a compile-time two-stage plan N = R1 * R2 (R1, R2 <= 16).
PLANS = {
    16: (4, 4), 24: (8, 3), 32: (8, 4), 48: (16, 3), 56: (8, 7), 64: (8, 8), 72: (8, 9),
    88: (8, 11), 96: (16, 6), 112: (16, 7), 128: (16, 8), 144: (16, 9), 176: (16, 11),
    192: (16, 12), 224: (16, 14), 256: (16, 16),
}
RADICES = [2, 3, 4, 5, 6, 7, 8, 9, 11, 12, 13, 14, 16]


def f32(v):
    s = repr(float(np.float32(v)))
    if "e" not in s and "." not in s:
        s += ".0"
    return s + "f"


def main():
    lines = ["// Generated by gen_twiddles.py -- do not edit.", "#pragma once", "",
             "namespace me {", ""]
    lines.append("// Two-stage plans N = R1 * R2 for the compile-time line FFTs.")
    lines.append("#define ME_FAST_LENGTHS(X) \\")
    items = [f"  X({n}, {r1}, {r2})" for n, (r1, r2) in sorted(PLANS.items())]
    lines.append(" \\\n".join(items))
    lines.append("")
    for n in sorted(PLANS):
        m = np.arange(n)
        ang = -2.0 * np.pi * m / n
        vals = ", ".join(f"{{{f32(np.cos(a))}, {f32(np.sin(a))}}}" for a in ang)
        lines.append(f"__device__ const float2 tw{n}[{n}] = {{{vals}}};")
    lines.append("")
    lines.append("// The second-stage twiddles of each plan in the order the threads read them:")
    lines.append("// twp<N>[r R1 + j] = tw<N>[(r j) mod N] (the same float32 values), so that the R1")
    lines.append("// threads of a line read R1 consecutive entries for each r.")
    for n, (r1, r2) in sorted(PLANS.items()):
        ms = [(r * j) % n for r in range(r2) for j in range(r1)]
        ang = [-2.0 * np.pi * m / n for m in ms]
        vals = ", ".join(f"{{{f32(np.cos(a))}, {f32(np.sin(a))}}}" for a in ang)
        lines.append(f"__device__ const float2 twp{n}[{r1 * r2}] = {{{vals}}};")
    lines.append("")
    lines.append("// cos / sin of 2 pi m / R for the register DFTs (m is a compile-time constant at")
    lines.append("// every call site after unrolling, so these fold to immediates)")
    lines.append("template <int R> struct RadixConst;")
    for r in RADICES:
        m = np.arange(r)
        c = ", ".join(f32(np.cos(2 * np.pi * k / r)) for k in m)
        s = ", ".join(f32(np.sin(2 * np.pi * k / r)) for k in m)
        lines.append(f"template <> struct RadixConst<{r}> {{")
        lines.append(f"  static __host__ __device__ __forceinline__ float c(int m) {{")
        lines.append(f"    constexpr float t[{r}] = {{{c}}};")
        lines.append("    return t[m];")
        lines.append("  }")
        lines.append(f"  static __host__ __device__ __forceinline__ float s(int m) {{")
        lines.append(f"    constexpr float t[{r}] = {{{s}}};")
        lines.append("    return t[m];")
        lines.append("  }")
        lines.append("};")
    lines.append("")
    lines.append("}  // namespace me")
    OUT.write_text("\n".join(lines) + "\n")
    return OUT


if __name__ == "__main__":
    print(main())
