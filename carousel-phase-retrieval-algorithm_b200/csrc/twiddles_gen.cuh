// generated by gen_twiddles.py: cos/sin(2*pi*k/32), k < 32
#pragma once
namespace cpra_b200 {
__host__ __device__ __forceinline__ constexpr double tw32_cos_d(int k) {
    switch (k & 31) {
        case 0: return 0x1.0000000000000p+0;
        case 1: return 0x1.f6297cff75cb0p-1;
        case 2: return 0x1.d906bcf328d46p-1;
        case 3: return 0x1.a9b66290ea1a3p-1;
        case 4: return 0x1.6a09e667f3bcdp-1;
        case 5: return 0x1.1c73b39ae68c9p-1;
        case 6: return 0x1.87de2a6aea964p-2;
        case 7: return 0x1.8f8b83c69a60dp-3;
        case 8: return 0x0.0p+0;
        case 9: return -0x1.8f8b83c69a608p-3;
        case 10: return -0x1.87de2a6aea962p-2;
        case 11: return -0x1.1c73b39ae68c6p-1;
        case 12: return -0x1.6a09e667f3bccp-1;
        case 13: return -0x1.a9b66290ea1a4p-1;
        case 14: return -0x1.d906bcf328d46p-1;
        case 15: return -0x1.f6297cff75cb0p-1;
        case 16: return -0x1.0000000000000p+0;
        case 17: return -0x1.f6297cff75cb0p-1;
        case 18: return -0x1.d906bcf328d47p-1;
        case 19: return -0x1.a9b66290ea1a5p-1;
        case 20: return -0x1.6a09e667f3bcep-1;
        case 21: return -0x1.1c73b39ae68c8p-1;
        case 22: return -0x1.87de2a6aea96dp-2;
        case 23: return -0x1.8f8b83c69a619p-3;
        case 24: return 0x0.0p+0;
        case 25: return 0x1.8f8b83c69a60cp-3;
        case 26: return 0x1.87de2a6aea967p-2;
        case 27: return 0x1.1c73b39ae68c5p-1;
        case 28: return 0x1.6a09e667f3bcbp-1;
        case 29: return 0x1.a9b66290ea1a3p-1;
        case 30: return 0x1.d906bcf328d44p-1;
        case 31: return 0x1.f6297cff75cafp-1;
        default: return 0;
    }
}
__host__ __device__ __forceinline__ constexpr double tw32_sin_d(int k) {
    switch (k & 31) {
        case 0: return 0x0.0p+0;
        case 1: return 0x1.8f8b83c69a60ap-3;
        case 2: return 0x1.87de2a6aea963p-2;
        case 3: return 0x1.1c73b39ae68c8p-1;
        case 4: return 0x1.6a09e667f3bccp-1;
        case 5: return 0x1.a9b66290ea1a3p-1;
        case 6: return 0x1.d906bcf328d46p-1;
        case 7: return 0x1.f6297cff75cb0p-1;
        case 8: return 0x1.0000000000000p+0;
        case 9: return 0x1.f6297cff75cb0p-1;
        case 10: return 0x1.d906bcf328d46p-1;
        case 11: return 0x1.a9b66290ea1a5p-1;
        case 12: return 0x1.6a09e667f3bcdp-1;
        case 13: return 0x1.1c73b39ae68c8p-1;
        case 14: return 0x1.87de2a6aea965p-2;
        case 15: return 0x1.8f8b83c69a617p-3;
        case 16: return 0x0.0p+0;
        case 17: return -0x1.8f8b83c69a60ep-3;
        case 18: return -0x1.87de2a6aea961p-2;
        case 19: return -0x1.1c73b39ae68c6p-1;
        case 20: return -0x1.6a09e667f3bccp-1;
        case 21: return -0x1.a9b66290ea1a3p-1;
        case 22: return -0x1.d906bcf328d44p-1;
        case 23: return -0x1.f6297cff75cafp-1;
        case 24: return -0x1.0000000000000p+0;
        case 25: return -0x1.f6297cff75cb0p-1;
        case 26: return -0x1.d906bcf328d45p-1;
        case 27: return -0x1.a9b66290ea1a5p-1;
        case 28: return -0x1.6a09e667f3bcep-1;
        case 29: return -0x1.1c73b39ae68c8p-1;
        case 30: return -0x1.87de2a6aea96ep-2;
        case 31: return -0x1.8f8b83c69a61bp-3;
        default: return 0;
    }
}
__host__ __device__ __forceinline__ constexpr float tw32_cos_f(int k) {
    switch (k & 31) {
        case 0: return 0x1.0000000000000p+0f;
        case 1: return 0x1.f6297c0000000p-1f;
        case 2: return 0x1.d906bc0000000p-1f;
        case 3: return 0x1.a9b6620000000p-1f;
        case 4: return 0x1.6a09e60000000p-1f;
        case 5: return 0x1.1c73b40000000p-1f;
        case 6: return 0x1.87de2a0000000p-2f;
        case 7: return 0x1.8f8b840000000p-3f;
        case 8: return 0x0.0p+0f;
        case 9: return -0x1.8f8b840000000p-3f;
        case 10: return -0x1.87de2a0000000p-2f;
        case 11: return -0x1.1c73b40000000p-1f;
        case 12: return -0x1.6a09e60000000p-1f;
        case 13: return -0x1.a9b6620000000p-1f;
        case 14: return -0x1.d906bc0000000p-1f;
        case 15: return -0x1.f6297c0000000p-1f;
        case 16: return -0x1.0000000000000p+0f;
        case 17: return -0x1.f6297c0000000p-1f;
        case 18: return -0x1.d906bc0000000p-1f;
        case 19: return -0x1.a9b6620000000p-1f;
        case 20: return -0x1.6a09e60000000p-1f;
        case 21: return -0x1.1c73b40000000p-1f;
        case 22: return -0x1.87de2a0000000p-2f;
        case 23: return -0x1.8f8b840000000p-3f;
        case 24: return 0x0.0p+0f;
        case 25: return 0x1.8f8b840000000p-3f;
        case 26: return 0x1.87de2a0000000p-2f;
        case 27: return 0x1.1c73b40000000p-1f;
        case 28: return 0x1.6a09e60000000p-1f;
        case 29: return 0x1.a9b6620000000p-1f;
        case 30: return 0x1.d906bc0000000p-1f;
        case 31: return 0x1.f6297c0000000p-1f;
        default: return 0;
    }
}
__host__ __device__ __forceinline__ constexpr float tw32_sin_f(int k) {
    switch (k & 31) {
        case 0: return 0x0.0p+0f;
        case 1: return 0x1.8f8b840000000p-3f;
        case 2: return 0x1.87de2a0000000p-2f;
        case 3: return 0x1.1c73b40000000p-1f;
        case 4: return 0x1.6a09e60000000p-1f;
        case 5: return 0x1.a9b6620000000p-1f;
        case 6: return 0x1.d906bc0000000p-1f;
        case 7: return 0x1.f6297c0000000p-1f;
        case 8: return 0x1.0000000000000p+0f;
        case 9: return 0x1.f6297c0000000p-1f;
        case 10: return 0x1.d906bc0000000p-1f;
        case 11: return 0x1.a9b6620000000p-1f;
        case 12: return 0x1.6a09e60000000p-1f;
        case 13: return 0x1.1c73b40000000p-1f;
        case 14: return 0x1.87de2a0000000p-2f;
        case 15: return 0x1.8f8b840000000p-3f;
        case 16: return 0x0.0p+0f;
        case 17: return -0x1.8f8b840000000p-3f;
        case 18: return -0x1.87de2a0000000p-2f;
        case 19: return -0x1.1c73b40000000p-1f;
        case 20: return -0x1.6a09e60000000p-1f;
        case 21: return -0x1.a9b6620000000p-1f;
        case 22: return -0x1.d906bc0000000p-1f;
        case 23: return -0x1.f6297c0000000p-1f;
        case 24: return -0x1.0000000000000p+0f;
        case 25: return -0x1.f6297c0000000p-1f;
        case 26: return -0x1.d906bc0000000p-1f;
        case 27: return -0x1.a9b6620000000p-1f;
        case 28: return -0x1.6a09e60000000p-1f;
        case 29: return -0x1.1c73b40000000p-1f;
        case 30: return -0x1.87de2a0000000p-2f;
        case 31: return -0x1.8f8b840000000p-3f;
        default: return 0;
    }
}
}  // namespace cpra_b200
