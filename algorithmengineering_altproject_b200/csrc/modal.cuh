// Modal (corner-Hadamard) form of the hex8 stiffness shared by the FP32 K(E)p kernels: the pattern of the
// 45 nonzeros of Kh = T^T Ke T / 64 and the x-y Hadamard stages (see k_matvec_modal.cu for the derivation).
#pragma once
#include <cuda_runtime.h>

namespace t3d {
namespace {

// modal index = component * 8 + mode, mode bit 0 = x, bit 1 = y, bit 2 = z (constant mode 0 unused)
// X(dst, src) for each of the 45 nonzeros, in the order of ModalKe::v
#define T3D_KH_PATTERN(X)                                                                          \
    /* normal strains: (0,x) (1,y) (2,z) */                                                        \
    X(1, 1) X(1, 10) X(1, 20) X(10, 1) X(10, 10) X(10, 20) X(20, 1) X(20, 10) X(20, 20)            \
    /* shears xy, xz, yz */                                                                        \
    X(9, 9) X(9, 2) X(2, 9) X(2, 2) X(17, 17) X(17, 4) X(4, 17) X(4, 4)                            \
    X(18, 18) X(18, 12) X(12, 18) X(12, 12)                                                        \
    /* bilinear pairs */                                                                           \
    X(3, 3) X(3, 22) X(22, 3) X(22, 22) X(11, 11) X(11, 21) X(21, 11) X(21, 21)                    \
    X(5, 5) X(5, 14) X(14, 5) X(14, 14)                                                            \
    /* bilinear triple (2,xy) (1,xz) (0,yz) */                                                     \
    X(19, 19) X(19, 13) X(19, 6) X(13, 19) X(13, 13) X(13, 6) X(6, 19) X(6, 13) X(6, 6)            \
    /* trilinear */                                                                                \
    X(7, 7) X(15, 15) X(23, 23)

struct KhEntry {
    int dst, src;
};
#define T3D_KH_ENTRY(d, s) {d, s},
constexpr KhEntry KH_PATTERN_HOST[45] = {T3D_KH_PATTERN(T3D_KH_ENTRY)};
#undef T3D_KH_ENTRY

// x-y Hadamard stage of one component on one node plane: corners (dx,dy) -> modes (i,j)
struct Modes2 {
    float m00, m10, m01, m11;
};

__device__ __forceinline__ Modes2 fwd2(float u00, float u10, float u01, float u11) {
    const float s0 = u00 + u10, d0 = u10 - u00, s1 = u01 + u11, d1 = u11 - u01;
    return Modes2{s0 + s1, d0 + d1, s1 - s0, d1 - d0};
}

// inverse x-y stage: modes (i,j) -> corner values (dx,dy) = sum s_x^i s_y^j w_ij
__device__ __forceinline__ void inv2(const Modes2& w, float& v00, float& v10, float& v01, float& v11) {
    const float p = w.m00 - w.m01, q = w.m10 - w.m11, pp = w.m00 + w.m01, qq = w.m10 + w.m11;
    v00 = p - q;
    v10 = p + q;
    v01 = pp - qq;
    v11 = pp + qq;
}

// The same two stages on components 0 and 1 at once (packed FP32x2 arithmetic, .x = component 0,
// .y = component 1); a - b is fma(b, -1, a), which is exact.
struct Modes2x2 {
    float2 m00, m10, m01, m11;
};
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ Modes2x2 fwd2x2(float2 u00, float2 u10, float2 u01, float2 u11) {
    const float2 s0 = add2(u00, u10), d0 = sub2(u10, u00), s1 = add2(u01, u11), d1 = sub2(u11, u01);
    return Modes2x2{add2(s0, s1), add2(d0, d1), sub2(s1, s0), sub2(d1, d0)};
}
__device__ __forceinline__ void inv2x2(const Modes2x2& w, float2& v00, float2& v10, float2& v01, float2& v11) {
    const float2 p = sub2(w.m00, w.m01), q = sub2(w.m10, w.m11), pp = add2(w.m00, w.m01), qq = add2(w.m10, w.m11);
    v00 = sub2(p, q);
    v10 = add2(p, q);
    v01 = sub2(pp, qq);
    v11 = add2(pp, qq);
}

}  // namespace
}  // namespace t3d
