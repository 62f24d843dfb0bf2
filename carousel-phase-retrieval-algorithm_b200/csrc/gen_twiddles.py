"""Writes twiddles_gen.cuh: constexpr cos/sin(2*pi*k/32), k < 32, for float and double
literals, the in-register butterfly constants of the line FFTs (every radix
R <= 32 uses W_R^j = W_32^(j*32/R)).  Values come from Python's math.cos/sin
in double and are printed as hex floats; exact zeros and ones are used on the
quadrant points.  Run: python gen_twiddles.py > twiddles_gen.cuh"""
import math

N = 32


def cs(k):
    if (4 * k) % N == 0:
        q = (4 * k) // N
        return [(1.0, 0.0), (0.0, 1.0), (-1.0, 0.0), (0.0, -1.0)][q]
    a = 2.0 * math.pi * k / N
    return math.cos(a), math.sin(a)


def f32(v):
    import struct
    return struct.unpack("f", struct.pack("f", v))[0]


print("// generated by gen_twiddles.py: cos/sin(2*pi*k/32), k < 32")
print("#pragma once")
print("namespace cpra_b200 {")
for fn, conv, suf, ty in (("tw32_cos_d", lambda v: v, "", "double"),
                          ("tw32_sin_d", lambda v: v, "", "double"),
                          ("tw32_cos_f", f32, "f", "float"),
                          ("tw32_sin_f", f32, "f", "float")):
    idx = 0 if "cos" in fn else 1
    print(f"__host__ __device__ __forceinline__ constexpr {ty} {fn}(int k) {{")
    print("    switch (k & 31) {")
    for k in range(N):
        print(f"        case {k}: return {float.hex(conv(cs(k)[idx]))}{suf};")
    print(f"        default: return 0;")
    print("    }")
    print("}")
print("}  // namespace cpra_b200")
