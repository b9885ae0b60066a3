// The 5x5 Gaussian's one-axis step, shared by the pre-filter kernel and the
// cost kernels that fuse it: [1 4 6 4 1]/16 in the symmetric form
// c*k2 + (a1+b1)*k1 + (a2+b2)*k0, each operation rounded as written.
#ifndef TDV_GAUSS5_CUH
#define TDV_GAUSS5_CUH

namespace tdv {

__device__ __forceinline__ float gauss5(float a2, float a1, float c, float b1, float b2) {
    float s = __fmul_rn(c, 0.375f);
    s = __fadd_rn(s, __fmul_rn(__fadd_rn(a1, b1), 0.25f));
    return __fadd_rn(s, __fmul_rn(__fadd_rn(a2, b2), 0.0625f));
}

}  // namespace tdv

#endif  // TDV_GAUSS5_CUH
