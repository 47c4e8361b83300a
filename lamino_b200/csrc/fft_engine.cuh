// Shared-memory mixed-radix FFT engine for the Toeplitz apply (sm_100a).
//
// A length-n transform (n = product of radices in {2,3,4,5,8,9}) runs as
// in-place decimation-in-frequency stages: stage s with radix r and block size
// B_s = n / (r_0 ... r_{s-1}) combines the r elements base + m j (m = B_s / r),
// applies an r-point DFT and the twiddles w_{B_s}^{n1 k}.  The output is left in
// digit-reversed position order, which is never undone: the Toeplitz spectra
// are stored in the same position order, and the inverse ("undo") runs the
// stages backwards (conjugate twiddles, then an inverse r-point DFT), taking
// positions back to natural order and returning n x (unnormalised).
//
// Transforms of zero-padded data (input length <= n/2) start with a radix-2
// stage whose second input is zero; it is folded into the load, and the matching
// last undo stage (outputs < n/2 only) into the store.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include <vector>

namespace lamino {

constexpr int FFT_MAX_STAGES = 16;

// Division of 0 <= x < 2^31 by a runtime d >= 1 as a multiply-high, an add and a
// shift: q = (umulhi(x, mul) + x) >> sh, sh = ceil(log2 d),
// mul = floor(2^32 (2^sh - d) / d) + 1 (the round-up method).
struct FastDiv {
    uint32_t mul = 1, sh = 0;
    static FastDiv make(uint32_t d) {
        FastDiv f;
        while ((1ull << f.sh) < d) ++f.sh;
        f.mul = (uint32_t)((((1ull << 32) * ((1ull << f.sh) - d)) / d) + 1);
        return f;
    }
    __device__ __forceinline__ int div(int x) const {
        return (int)((__umulhi((uint32_t)x, mul) + (uint32_t)x) >> sh);
    }
};

struct FftLen {  // POD, passed by value to kernels
    int n, ns;
    int radix[FFT_MAX_STAGES];
    int bsz[FFT_MAX_STAGES];
    // per stage: division by the offsets per block (B / R), the butterflies per
    // pencil (n / R) and the blocks per pencil (n / B)
    FastDiv dm[FFT_MAX_STAGES], dnb[FFT_MAX_STAGES], dblk[FFT_MAX_STAGES];
    const float2 *tw;  // exp(-2 pi i e / n), e in [0, n)
};

// Bulk prefetch of [p, p + bytes) into L2 (cp.async.bulk.prefetch.L2, no
// multicast): the range is shrunk inward to 16-byte boundaries, so only bytes
// of the given range are touched.
__device__ __forceinline__ void prefetch_l2(const void *p, size_t bytes) {
    const uintptr_t a = (reinterpret_cast<uintptr_t>(p) + 15) & ~uintptr_t(15);
    const uintptr_t e = (reinterpret_cast<uintptr_t>(p) + bytes) & ~uintptr_t(15);
    if (e > a)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"((unsigned)(e - a)) : "memory");
}

// Complex arithmetic on Blackwell's packed FP32 pair instructions (add / mul /
// fma .f32x2: one instruction for both halves of a float2, per component the
// same rounding as the scalar operation).
__device__ __forceinline__ float2 c_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 c_sub(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 c_mul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 c_mulc(float2 a, float2 b) {  // a * conj(b)
    return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}
__device__ __forceinline__ float2 c_scale(float2 a, float s) { return __fmul2_rn(a, make_float2(s, s)); }
// a (c + i s) for constants c, s: one packed product and two scalar FMAs
__device__ __forceinline__ float2 c_mul_k(float2 a, float c, float s) {
    const float2 t = __fmul2_rn(a, make_float2(c, c));
    return make_float2(fmaf(-s, a.y, t.x), fmaf(s, a.x, t.y));
}
// s a + b for real s
__device__ __forceinline__ float2 c_fma(float s, float2 a, float2 b) { return __ffma2_rn(make_float2(s, s), a, b); }
// multiply by -i (forward) or +i (inverse)
template <bool INV>
__device__ __forceinline__ float2 c_rot(float2 a) {
    return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}
// m + (-i) s d and m - (-i) s d (forward; +i for the inverse), s real: the
// rotation swaps the halves, so these run as scalar FMAs.
template <bool INV>
__device__ __forceinline__ void c_rot_pm(float2 m, float2 d, float s, float2 &plus, float2 &minus) {
    if constexpr (!INV) {
        plus = make_float2(fmaf(s, d.y, m.x), fmaf(-s, d.x, m.y));
        minus = make_float2(fmaf(-s, d.y, m.x), fmaf(s, d.x, m.y));
    } else {
        plus = make_float2(fmaf(-s, d.y, m.x), fmaf(s, d.x, m.y));
        minus = make_float2(fmaf(s, d.y, m.x), fmaf(-s, d.x, m.y));
    }
}

template <bool INV>
__device__ __forceinline__ void dft3(float2 &x0, float2 &x1, float2 &x2) {
    const float c = -0.5f, s = 0.86602540378443864676f;
    float2 t = c_add(x1, x2);
    float2 d = c_sub(x1, x2);
    float2 y0 = c_add(x0, t);
    float2 m = c_fma(c, t, x0);
    x0 = y0;
    c_rot_pm<INV>(m, d, s, x1, x2);  // m -/+ i s d
}

template <bool INV>
__device__ __forceinline__ void dft4(float2 &x0, float2 &x1, float2 &x2, float2 &x3) {
    float2 a = c_add(x0, x2), b = c_sub(x0, x2);
    float2 c = c_add(x1, x3), e = c_sub(x1, x3);
    x0 = c_add(a, c);
    x2 = c_sub(a, c);
    c_rot_pm<INV>(b, e, 1.f, x1, x3);  // b -/+ i e
}

template <bool INV>
__device__ __forceinline__ void dft5(float2 (&v)[5]) {
    const float c1 = 0.30901699437494742410f, c2 = -0.80901699437494742410f;
    const float s1 = 0.95105651629515357212f, s2 = 0.58778525229247312917f;
    float2 a1 = c_add(v[1], v[4]), b1 = c_sub(v[1], v[4]);
    float2 a2 = c_add(v[2], v[3]), b2 = c_sub(v[2], v[3]);
    float2 y0 = c_add(v[0], c_add(a1, a2));
    float2 m1 = c_fma(c2, a2, c_fma(c1, a1, v[0]));
    float2 m2 = c_fma(c1, a2, c_fma(c2, a1, v[0]));
    // -i (s1 b1 + s2 b2) and -i (s2 b1 - s1 b2) for the forward transform
    float2 p1 = c_fma(s2, b2, c_scale(b1, s1));
    float2 p2 = c_fma(-s1, b2, c_scale(b1, s2));
    v[0] = y0;
    c_rot_pm<INV>(m1, p1, 1.f, v[1], v[4]);
    c_rot_pm<INV>(m2, p2, 1.f, v[2], v[3]);
}

template <bool INV>
__device__ __forceinline__ void dft8(float2 (&v)[8]) {
    // y[k] = E[k mod 4] + W8^k O[k mod 4], E/O = 4-point DFTs of even/odd inputs
    float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    float2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4<INV>(e0, e1, e2, e3);
    dft4<INV>(o0, o1, o2, o3);
    const float h = 0.70710678118654752440f;
    // W8^1 o = h q1 with q1 = o -/+ i o (fwd / inv), W8^2 o = -/+ i o,
    // W8^3 o = h q3 with q3 = -o -/+ i o
    const float2 q1 = INV ? make_float2(o1.x - o1.y, o1.x + o1.y) : make_float2(o1.x + o1.y, o1.y - o1.x);
    const float2 q3 = INV ? make_float2(-(o3.x + o3.y), o3.x - o3.y) : make_float2(o3.y - o3.x, -(o3.x + o3.y));
    v[0] = c_add(e0, o0);
    v[4] = c_sub(e0, o0);
    v[1] = c_fma(h, q1, e1);
    v[5] = c_fma(-h, q1, e1);
    c_rot_pm<INV>(e2, o2, 1.f, v[2], v[6]);
    v[3] = c_fma(h, q3, e3);
    v[7] = c_fma(-h, q3, e3);
}

template <bool INV>
__device__ __forceinline__ void dft9(float2 (&v)[9]) {
    // j = j1 + 3 j2, k = 3 k1 + k2: inner 3-point DFTs over j2, twiddle W9^{j1 k2}, outer over j1
    float2 a[3][3];
#pragma unroll
    for (int j1 = 0; j1 < 3; ++j1) {
        a[j1][0] = v[j1];
        a[j1][1] = v[j1 + 3];
        a[j1][2] = v[j1 + 6];
        dft3<INV>(a[j1][0], a[j1][1], a[j1][2]);
    }
    const float c1 = 0.76604444311897803520f, s1 = 0.64278760968653932632f;   // W9^1
    const float c2 = 0.17364817766693034885f, s2 = 0.98480775301220805936f;   // W9^2
    const float c4 = -0.93969262078590838405f, s4 = 0.34202014332566873304f;  // W9^4
    const float sg = INV ? 1.f : -1.f;
    a[1][1] = c_mul_k(a[1][1], c1, sg * s1);
    a[1][2] = c_mul_k(a[1][2], c2, sg * s2);
    a[2][1] = c_mul_k(a[2][1], c2, sg * s2);
    a[2][2] = c_mul_k(a[2][2], c4, sg * s4);
#pragma unroll
    for (int k2 = 0; k2 < 3; ++k2) {
        float2 y0 = a[0][k2], y1 = a[1][k2], y2 = a[2][k2];
        dft3<INV>(y0, y1, y2);
        v[k2] = y0;
        v[3 + k2] = y1;
        v[6 + k2] = y2;
    }
}

// cos / sin of 2 pi m / 27, m = 0..16 (the twiddles inside the 27-point DFT);
// called with compile-time m, so the values fold into the instructions
__host__ __device__ constexpr float w27c(int m) {
    constexpr float t[17] = {1.f,
                             0.97304487057982380627f,  0.89363264032341227505f,  0.76604444311897801345f,
                             0.59715859170278617896f,  0.39607976603915689973f,  0.17364817766693041445f,
                             -0.05814482891047577373f, -0.28680323271109020578f, -0.49999999999999977796f,
                             -0.68624163786873348947f, -0.83548781141293626540f, -0.93969262078590831688f,
                             -0.99323835774194302317f, -0.99323835774194302317f, -0.93969262078590853893f,
                             -0.83548781141293648744f};
    return t[m];
}
__host__ __device__ constexpr float w27s(int m) {
    constexpr float t[17] = {0.f,
                             0.23061587074244016549f,  0.44879918020046216665f,  0.64278760968653925190f,
                             0.80212319275504373461f,  0.91821610688027399672f,  0.98480775301220802032f,
                             0.99830815827126817563f,  0.95798951231548890028f,  0.86602540378443870761f,
                             0.72737364157304884582f,  0.54950897807080623103f,  0.34202014332566887944f,
                             0.11609291412522992903f,  -0.11609291412523012332f, -0.34202014332566821331f,
                             -0.54950897807080600899f};
    return t[m];
}

// 27-point DFT in registers: j = 3 j2 + j1, k = k1 + 9 k2; 9-point DFTs over
// j2, twiddles W27^{j1 k1}, 3-point DFTs over j1.  Natural order in and out.
template <bool INV>
__device__ __forceinline__ void dft27(float2 (&v)[27]) {
    float2 a[3][9];
#pragma unroll
    for (int j1 = 0; j1 < 3; ++j1) {
#pragma unroll
        for (int j2 = 0; j2 < 9; ++j2) a[j1][j2] = v[3 * j2 + j1];
        dft9<INV>(a[j1]);
    }
    const float sg = INV ? 1.f : -1.f;
#pragma unroll
    for (int k1 = 1; k1 < 9; ++k1) {
        a[1][k1] = c_mul_k(a[1][k1], w27c(k1), sg * w27s(k1));
        a[2][k1] = c_mul_k(a[2][k1], w27c(2 * k1), sg * w27s(2 * k1));
    }
#pragma unroll
    for (int k1 = 0; k1 < 9; ++k1) {
        float2 y0 = a[0][k1], y1 = a[1][k1], y2 = a[2][k1];
        dft3<INV>(y0, y1, y2);
        v[k1] = y0;
        v[k1 + 9] = y1;
        v[k1 + 18] = y2;
    }
}

// v[k] *= b w^{e k} for k = 0..26 (conjugated for the inverse), w^e = tw[e]:
// with k = k0 + 3 k1 + 9 k2 every factor is at most a few products from the
// table values tw[e], tw[3e], tw[9e] (3 table loads for 27 twiddles).
template <bool INV>
__device__ __forceinline__ void twiddle27(const float2 *__restrict__ tw, int e, float2 b, float2 (&v)[27]) {
    const float2 z = __ldg(tw + e), z3 = __ldg(tw + 3 * e), z9 = __ldg(tw + 9 * e);
    float2 p0[3];
    p0[0] = b;
    p0[1] = c_mul(b, z);
    p0[2] = c_mul(p0[1], z);
    const float2 z6 = c_mul(z3, z3), z18 = c_mul(z9, z9);
#pragma unroll
    for (int k1 = 0; k1 < 3; ++k1) {
#pragma unroll
        for (int k0 = 0; k0 < 3; ++k0) {
            const float2 p = k1 == 0 ? p0[k0] : c_mul(p0[k0], k1 == 1 ? z3 : z6);
#pragma unroll
            for (int k2 = 0; k2 < 3; ++k2) {
                const int k = k0 + 3 * k1 + 9 * k2;
                const float2 t = k2 == 0 ? p : c_mul(p, k2 == 1 ? z9 : z18);
                v[k] = INV ? c_mulc(v[k], t) : c_mul(v[k], t);
            }
        }
    }
}

// w^k for k = 1..R-1 from two table loads (w = tw[e], w4 = tw[4e] when R > 4),
// every power at most two complex products away from a loaded value.
template <int R>
__device__ __forceinline__ void twiddle_powers(const float2 *__restrict__ tw, int e, float2 (&w)[R]) {
    w[1] = __ldg(tw + e);
    if constexpr (R > 2) w[2] = c_mul(w[1], w[1]);
    if constexpr (R > 3) w[3] = c_mul(w[2], w[1]);
    if constexpr (R > 4) {
        w[4] = __ldg(tw + 4 * e);
        if constexpr (R > 5) w[5] = c_mul(w[4], w[1]);
        if constexpr (R > 6) w[6] = c_mul(w[4], w[2]);
        if constexpr (R > 7) w[7] = c_mul(w[4], w[3]);
        if constexpr (R > 8) w[8] = c_mul(w[4], w[4]);
    }
}

template <int R, bool INV>
__device__ __forceinline__ void dft_small(float2 (&v)[R]) {
    if constexpr (R == 2) {
        float2 a = v[0];
        v[0] = c_add(a, v[1]);
        v[1] = c_sub(a, v[1]);
    } else if constexpr (R == 3) {
        dft3<INV>(v[0], v[1], v[2]);
    } else if constexpr (R == 4) {
        dft4<INV>(v[0], v[1], v[2], v[3]);
    } else if constexpr (R == 5) {
        dft5<INV>(v);
    } else if constexpr (R == 8) {
        dft8<INV>(v);
    } else {
        static_assert(R == 9, "unsupported radix");
        dft9<INV>(v);
    }
}

// One stage over P pencils of length n (pencil stride ps) in shared memory, the
// runtime-length counterpart of fft_stage_fixed: the butterfly index is split with
// multiply-high divisions, the twiddles come from two table loads and products,
// and with fewer than 16 offsets per odd-sized block the blocks run fastest (lanes
// B apart, distinct banks).
template <int R, bool INV>
__device__ __forceinline__ void fft_stage(float2 *__restrict__ data, int P, int ps, int n, int B,
                                          const float2 *__restrict__ tw, FastDiv dm, FastDiv dnb, FastDiv dblk,
                                          int tid, int nth) {
    const int m = B / R;
    const int nb = n / R;
    const int ts = n / B;
    const int nblk = ts;
    const bool b_fast = (m > 1) && (m < 16) && (B & 1);
    const int total = P * nb;
    for (int t = tid; t < total; t += nth) {
        const int pen = dnb.div(t);
        const int u = t - pen * nb;
        int b, n1;
        if (b_fast) {
            n1 = dblk.div(u);
            b = u - n1 * nblk;
        } else {
            b = dm.div(u);
            n1 = u - b * m;
        }
        float2 *base = data + pen * ps + b * B + n1;
        float2 v[R];
        if constexpr (!INV) {
#pragma unroll
            for (int j = 0; j < R; ++j) v[j] = base[m * j];
            dft_small<R, false>(v);
            if (n1 != 0) {
                float2 w[R];
                twiddle_powers<R>(tw, n1 * ts, w);
#pragma unroll
                for (int k = 1; k < R; ++k) v[k] = c_mul(v[k], w[k]);
            }
#pragma unroll
            for (int k = 0; k < R; ++k) base[m * k] = v[k];
        } else {
#pragma unroll
            for (int k = 0; k < R; ++k) v[k] = base[m * k];
            if (n1 != 0) {
                float2 w[R];
                twiddle_powers<R>(tw, n1 * ts, w);
#pragma unroll
                for (int k = 1; k < R; ++k) v[k] = c_mulc(v[k], w[k]);
            }
            dft_small<R, true>(v);
#pragma unroll
            for (int j = 0; j < R; ++j) base[m * j] = v[j];
        }
    }
}

template <bool INV>
__device__ __forceinline__ void fft_stage_rt(const FftLen &F, int s, float2 *data, int P, int ps, int tid,
                                             int nth) {
    const int n = F.n, B = F.bsz[s];
    const FastDiv dm = F.dm[s], dnb = F.dnb[s], dblk = F.dblk[s];
    switch (F.radix[s]) {
        case 2: fft_stage<2, INV>(data, P, ps, n, B, F.tw, dm, dnb, dblk, tid, nth); break;
        case 3: fft_stage<3, INV>(data, P, ps, n, B, F.tw, dm, dnb, dblk, tid, nth); break;
        case 4: fft_stage<4, INV>(data, P, ps, n, B, F.tw, dm, dnb, dblk, tid, nth); break;
        case 5: fft_stage<5, INV>(data, P, ps, n, B, F.tw, dm, dnb, dblk, tid, nth); break;
        case 8: fft_stage<8, INV>(data, P, ps, n, B, F.tw, dm, dnb, dblk, tid, nth); break;
        default: fft_stage<9, INV>(data, P, ps, n, B, F.tw, dm, dnb, dblk, tid, nth); break;
    }
}

// forward DIF stages s_begin .. ns-1 (caller synchronises before the call)
__device__ __forceinline__ void fft_forward(float2 *data, int P, int ps, const FftLen &F, int s_begin, int tid,
                                            int nth) {
    for (int s = s_begin; s < F.ns; ++s) {
        fft_stage_rt<false>(F, s, data, P, ps, tid, nth);
        __syncthreads();
    }
}

// undo stages ns-1 .. s_end (caller synchronises before the call)
__device__ __forceinline__ void fft_inverse(float2 *data, int P, int ps, const FftLen &F, int s_end, int tid,
                                            int nth) {
    for (int s = F.ns - 1; s >= s_end; --s) {
        fft_stage_rt<true>(F, s, data, P, ps, tid, nth);
        __syncthreads();
    }
}

// ---- compile-time schedules for the lengths of the common problem sizes ----
// (729 = packed n3 transform and 1458 = n1 transform of a 721-voxel axis; 144 =
// n2 transform of a 71-voxel axis; 180, 360 = n1 transforms of the 90- and
// 180-voxel lateral axes of 64- and 128-wide reconstructions; 20, 48, 64, 90 =
// n2 transforms of their 10- to 44-voxel thickness axes; 540 and 750 run in two
// register stages instead).
// Each equals the runtime schedule fft_schedule(N, true), so the DIF output
// positions are the same either way.  Other lengths use the runtime path above.
constexpr int CT_MAX_STAGES = 6;
template <int N>
struct CtSched {
    static constexpr int ns = 0;
    static constexpr int r[CT_MAX_STAGES] = {0, 0, 0, 0, 0, 0};
};
template <>
struct CtSched<729> {
    static constexpr int ns = 3;
    static constexpr int r[CT_MAX_STAGES] = {9, 9, 9, 0, 0, 0};
};
template <>
struct CtSched<1458> {
    static constexpr int ns = 4;
    static constexpr int r[CT_MAX_STAGES] = {2, 9, 9, 9, 0, 0};
};
template <>
struct CtSched<144> {
    static constexpr int ns = 3;
    static constexpr int r[CT_MAX_STAGES] = {2, 8, 9, 0, 0, 0};
};
template <>
struct CtSched<180> {
    static constexpr int ns = 4;
    static constexpr int r[CT_MAX_STAGES] = {2, 2, 9, 5, 0, 0};
};
template <>
struct CtSched<360> {
    static constexpr int ns = 4;
    static constexpr int r[CT_MAX_STAGES] = {2, 4, 9, 5, 0, 0};
};
// n2 transforms of the 10-, 22-, 32- and 44-voxel thickness axes
template <>
struct CtSched<20> {
    static constexpr int ns = 3;
    static constexpr int r[CT_MAX_STAGES] = {2, 2, 5, 0, 0, 0};
};
template <>
struct CtSched<48> {
    static constexpr int ns = 3;
    static constexpr int r[CT_MAX_STAGES] = {2, 8, 3, 0, 0, 0};
};
template <>
struct CtSched<64> {
    static constexpr int ns = 3;
    static constexpr int r[CT_MAX_STAGES] = {2, 4, 8, 0, 0, 0};
};
template <>
struct CtSched<90> {
    static constexpr int ns = 3;
    static constexpr int r[CT_MAX_STAGES] = {2, 9, 5, 0, 0, 0};
};

// Schedules of the packed row transforms (no zero-padded lead stage): the
// packed half lengths 90 and 180 of the 180- and 360-long n3 embeddings (270
// and 375 run in two register stages).  Each equals fft_schedule(N, false).
template <int N>
struct CtRowSched {
    static constexpr int ns = 0;
    static constexpr int r[CT_MAX_STAGES] = {0, 0, 0, 0, 0, 0};
};
template <>
struct CtRowSched<90> {
    static constexpr int ns = 3;
    static constexpr int r[CT_MAX_STAGES] = {2, 9, 5, 0, 0, 0};
};
template <>
struct CtRowSched<180> {
    static constexpr int ns = 3;
    static constexpr int r[CT_MAX_STAGES] = {4, 9, 5, 0, 0, 0};
};

// block size before stage s of schedule SC (length N)
template <int N, class SC>
__host__ __device__ constexpr int ct_block(int s) {
    int b = N;
    for (int i = 0; i < s; ++i) b /= SC::r[i];
    return b;
}

// one stage with compile-time radix, length and block size
template <int R, int N, int B, bool INV>
__device__ __forceinline__ void fft_stage_fixed(float2 *__restrict__ data, int P, int ps,
                                                const float2 *__restrict__ tw, int tid, int nth) {
    constexpr int m = B / R;
    constexpr int nb = N / R;
    constexpr int ts = N / B;
    // Thread order over the (block b, offset n1) butterflies: n1 fastest reads
    // consecutive addresses, but with fewer than 16 offsets per block a half-warp
    // spans blocks B apart and collides in the shared-memory banks; with b fastest
    // the lanes are B apart, all distinct banks when B is odd (and they share
    // their twiddles).
    constexpr bool b_fast = (m > 1) && (m < 16) && (B % 2 == 1);
    constexpr int nblk = N / B;
    const int total = P * nb;
    for (int t = tid; t < total; t += nth) {
        const int pen = t / nb;
        const int u = t - pen * nb;
        const int b = b_fast ? u % nblk : u / m;
        const int n1 = b_fast ? u / nblk : u - b * m;
        float2 *base = data + pen * ps + b * B + n1;
        float2 v[R];
        if constexpr (!INV) {
#pragma unroll
            for (int j = 0; j < R; ++j) v[j] = base[m * j];
            dft_small<R, false>(v);
            if constexpr (m > 1) {
                if (n1 != 0) {
                    float2 w[R];
                    twiddle_powers<R>(tw, n1 * ts, w);
#pragma unroll
                    for (int k = 1; k < R; ++k) v[k] = c_mul(v[k], w[k]);
                }
            }
#pragma unroll
            for (int k = 0; k < R; ++k) base[m * k] = v[k];
        } else {
#pragma unroll
            for (int k = 0; k < R; ++k) v[k] = base[m * k];
            if constexpr (m > 1) {
                if (n1 != 0) {
                    float2 w[R];
                    twiddle_powers<R>(tw, n1 * ts, w);
#pragma unroll
                    for (int k = 1; k < R; ++k) v[k] = c_mulc(v[k], w[k]);
                }
            }
            dft_small<R, true>(v);
#pragma unroll
            for (int j = 0; j < R; ++j) base[m * j] = v[j];
        }
    }
}

// stages S .. SC::ns - 1 of schedule SC, each followed by a barrier
template <int N, int S, class SC = CtSched<N>>
__device__ __forceinline__ void ct_forward(float2 *data, int P, int ps, const float2 *tw, int tid, int nth) {
    if constexpr (S < SC::ns) {
        fft_stage_fixed<SC::r[S], N, ct_block<N, SC>(S), false>(data, P, ps, tw, tid, nth);
        __syncthreads();
        ct_forward<N, S + 1, SC>(data, P, ps, tw, tid, nth);
    }
}

// undo stages S, S-1, ..., S_END
template <int N, int S, int S_END, class SC = CtSched<N>>
__device__ __forceinline__ void ct_inverse(float2 *data, int P, int ps, const float2 *tw, int tid, int nth) {
    if constexpr (S >= S_END) {
        fft_stage_fixed<SC::r[S], N, ct_block<N, SC>(S), true>(data, P, ps, tw, tid, nth);
        __syncthreads();
        ct_inverse<N, S - 1, S_END, SC>(data, P, ps, tw, tid, nth);
    }
}

// Transforms of length 1458 (schedule 2, 9, 9, 9) whose input is zero from 729 on
// and of which only outputs below 729 are kept: the zero-padded radix-2 stage and
// the first radix-9 stage (two blocks of 729, 81 offsets each) run in registers
// between the caller's loads and shared memory, and their inverses between
// shared memory and the caller's stores, two round trips through shared memory
// fewer each way.  Thread (c, n) of 3 x 81 handles values n + 81 j of row c of
// sm (rows 1458 apart); rows.get(c, i) gives input i (zero past the data),
// rows.want(i) / rows.put(c, i, v) take output i.  tw: the 1458-point table.
constexpr int F1458_OFS = 81;

template <class Rows>
__device__ __forceinline__ void fft1458_load(const Rows &rows, const float2 *__restrict__ tw,
                                             float2 *__restrict__ sm, int tid) {
    if (tid >= 3 * F1458_OFS) return;
    const int c = tid / F1458_OFS, n = tid - c * F1458_OFS;
    float2 x[9], u[9];
#pragma unroll
    for (int j = 0; j < 9; ++j) x[j] = rows.get(c, n + F1458_OFS * j);
    // radix-2 stage over the zero-padded half: block 0 = x, block 1 = x w^i
#pragma unroll
    for (int j = 0; j < 9; ++j) u[j] = c_mul(x[j], __ldg(tw + n + F1458_OFS * j));
    dft_small<9, false>(x);
    dft_small<9, false>(u);
    if (n != 0) {
        float2 w[9];
        twiddle_powers<9>(tw, 2 * n, w);
#pragma unroll
        for (int k = 1; k < 9; ++k) {
            x[k] = c_mul(x[k], w[k]);
            u[k] = c_mul(u[k], w[k]);
        }
    }
    float2 *s = sm + c * 1458 + n;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        s[F1458_OFS * k] = x[k];
        s[729 + F1458_OFS * k] = u[k];
    }
}

template <class Rows>
__device__ __forceinline__ void fft1458_store(const Rows &rows, const float2 *__restrict__ tw,
                                              const float2 *__restrict__ sm, int tid) {
    if (tid >= 3 * F1458_OFS) return;
    const int c = tid / F1458_OFS, n = tid - c * F1458_OFS;
    const float2 *s = sm + c * 1458 + n;
    float2 a[9], b[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        a[k] = s[F1458_OFS * k];
        b[k] = s[729 + F1458_OFS * k];
    }
    if (n != 0) {
        float2 w[9];
        twiddle_powers<9>(tw, 2 * n, w);
#pragma unroll
        for (int k = 1; k < 9; ++k) {
            a[k] = c_mulc(a[k], w[k]);
            b[k] = c_mulc(b[k], w[k]);
        }
    }
    dft_small<9, true>(a);
    dft_small<9, true>(b);
#pragma unroll
    for (int j = 0; j < 9; ++j) {
        const int i = n + F1458_OFS * j;
        if (rows.want(i)) rows.put(c, i, c_add(a[j], c_mulc(b[j], __ldg(tw + i))));
    }
}

// The same register stages for a runtime length L (schedule 2, R1, ...): the
// zero-padded radix-2 stage and the first radix-R1 stage (two blocks of L / 2,
// m1 = L / (2 R1) offsets each) between the caller's loads / stores and shared
// memory; rows of sm are ps apart, items (c, n) of 3 x m1 are spread over the
// nth threads.  The caller runs stages 2 .. ns-1 (fft_forward / fft_inverse).
template <int R1, class Rows>
__device__ __forceinline__ void fftlead_load(const Rows &rows, const float2 *__restrict__ tw, float2 *__restrict__ sm,
                                             int L, int ps, int tid, int nth) {
    const int half = L / 2, m1 = half / R1;
    for (int t = tid; t < 3 * m1; t += nth) {
        const int c = t / m1, n = t - c * m1;
        float2 x[R1], u[R1];
#pragma unroll
        for (int j = 0; j < R1; ++j) x[j] = rows.get(c, n + m1 * j);
#pragma unroll
        for (int j = 0; j < R1; ++j) u[j] = c_mul(x[j], __ldg(tw + n + m1 * j));
        dft_small<R1, false>(x);
        dft_small<R1, false>(u);
        if (n != 0) {
            float2 w[R1];
            twiddle_powers<R1>(tw, 2 * n, w);
#pragma unroll
            for (int k = 1; k < R1; ++k) {
                x[k] = c_mul(x[k], w[k]);
                u[k] = c_mul(u[k], w[k]);
            }
        }
        float2 *sp = sm + c * ps + n;
#pragma unroll
        for (int k = 0; k < R1; ++k) {
            sp[m1 * k] = x[k];
            sp[half + m1 * k] = u[k];
        }
    }
}

template <int R1, class Rows>
__device__ __forceinline__ void fftlead_store(const Rows &rows, const float2 *__restrict__ tw,
                                              const float2 *__restrict__ sm, int L, int ps, int tid, int nth) {
    const int half = L / 2, m1 = half / R1;
    for (int t = tid; t < 3 * m1; t += nth) {
        const int c = t / m1, n = t - c * m1;
        const float2 *sp = sm + c * ps + n;
        float2 a[R1], b[R1];
#pragma unroll
        for (int k = 0; k < R1; ++k) {
            a[k] = sp[m1 * k];
            b[k] = sp[half + m1 * k];
        }
        if (n != 0) {
            float2 w[R1];
            twiddle_powers<R1>(tw, 2 * n, w);
#pragma unroll
            for (int k = 1; k < R1; ++k) {
                a[k] = c_mulc(a[k], w[k]);
                b[k] = c_mulc(b[k], w[k]);
            }
        }
        dft_small<R1, true>(a);
        dft_small<R1, true>(b);
#pragma unroll
        for (int j = 0; j < R1; ++j) {
            const int i = n + m1 * j;
            if (rows.want(i)) rows.put(c, i, c_add(a[j], c_mulc(b[j], __ldg(tw + i))));
        }
    }
}

// dispatch on the runtime first radix after the lead 2
template <bool STORE, class Rows>
__device__ __forceinline__ void fftlead_any(const Rows &rows, const FftLen &F, float2 *sm, int ps, int tid,
                                            int nth) {
#define LAMINO_LEAD_CASE(R)                                                       \
    case R:                                                                       \
        if constexpr (STORE) fftlead_store<R>(rows, F.tw, sm, F.n, ps, tid, nth); \
        else fftlead_load<R>(rows, F.tw, sm, F.n, ps, tid, nth);                  \
        break;
    switch (F.radix[1]) {
        LAMINO_LEAD_CASE(2)
        LAMINO_LEAD_CASE(3)
        LAMINO_LEAD_CASE(4)
        LAMINO_LEAD_CASE(5)
        LAMINO_LEAD_CASE(8)
        default: LAMINO_LEAD_CASE(9)
    }
#undef LAMINO_LEAD_CASE
}

// Forward / inverse with a compile-time schedule when N != 0, else the runtime one.
template <int N, int S_BEGIN>
__device__ __forceinline__ void fft_fwd_any(float2 *data, int P, int ps, const FftLen &F, int tid, int nth) {
    if constexpr (N == 0) fft_forward(data, P, ps, F, S_BEGIN, tid, nth);
    else ct_forward<N, S_BEGIN>(data, P, ps, F.tw, tid, nth);
}
template <int N, int S_END>
__device__ __forceinline__ void fft_inv_any(float2 *data, int P, int ps, const FftLen &F, int tid, int nth) {
    if constexpr (N == 0) fft_inverse(data, P, ps, F, S_END, tid, nth);
    else ct_inverse<N, CtSched<N>::ns - 1, S_END>(data, P, ps, F.tw, tid, nth);
}

// ---- host-side schedule ----
// Radix schedule for length n; lead2 puts a radix-2 stage first (zero-padded data).
std::vector<int> fft_schedule(int n, bool lead2);
// natural frequency k -> DIF output position
std::vector<int> fft_positions(int n, const std::vector<int> &radix);
// smallest even 2,3,5-smooth length >= n (defined with the NUFFT plans)
int64_t next_smooth_even(int64_t n);

}  // namespace lamino
