// learned.cu — the learned absorbing strip and the kernels that train it.
//
// A model built with pml = 0 has no absorbing layer: its computed region
// ends at the reference's 5-cell zero frame, which reflects.  The learned
// strip takes the outer `width` cells of the computed region (width 6 for the
// 256^3 configuration, against a 20-cell split-field PML) and, after every
// step, adds to each of its cells a correction of the 9 fields predicted by
// a small MLP from the cell's neighbourhood:
//   inputs (252): the 9 fields at the 27 cells of its 3x3x3 neighbourhood
//     (velocities times the local impedance rho*vp, so that all 243 values
//     share the units of stress), divided by their RMS s; the cell's vp, vs,
//     rho over 3000 m/s, 1732 m/s, 2000 kg/m^3; per axis, the depth into the
//     strip (1..width over width, 0 off the strip band) and the side (-1 low,
//     +1 high, 0 off the band);
//   network: 252 -> 64 -> 64 -> 9, GELU after both hidden layers;
//   output: 9 corrections in units of s (velocities divided back by rho*vp),
//     so that the correction scales with the wavefield, as the physics does,
//     scaled down where needed so that no correction raises its cell's
//     energy (k_strip_tc).
// Parameters, 20 937 floats: W1 [252][64], b1, W2 [64][64], b2, W3 [64][9], b3.
//
// Inference (k_strip_tc) runs the three layers on the tensor cores
// (tcgen05.mma kind::f16: FP16 operands in shared memory, FP32 accumulators
// in tensor memory), 128 strip cells per tile.  The strip is cut into boxes
// of at most 128 cells (32 x 2 x 2 on the z and y faces, width x 4 x 5 on the
// x faces for width 6); a box's fields and their one-cell halo are staged in
// shared memory with coalesced loads, with each staged cell's sums of squares,
// and two threads build a cell's 252 inputs from there into row t of the A
// operand.
// Each CTA (one per SM) holds the weights once and runs three groups of 256
// threads that work on alternate tiles, so one group's loads overlap the
// other's tensor-core and epilogue work; two threads share each row.  The
// hidden layers' GELU uses a Chebyshev fit of erfc (Numerical Recipes erfcc,
// fractional error < 1.2e-7) with the exponential on the special-function unit.
//
// Training (sgfd_mlp_train) runs minibatch Adam with hand-written kernels:
// a tiled FP32 GEMM, bias + GELU, the output loss (mean squared error over the
// 9 outputs), the GELU backward, column sums and the Adam update.  The
// gradients are checked against a CPU restatement in the tests.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include <cuda_fp16.h>

#include "solver.h"
#include "strip_tiles.h"

using namespace sgfd;

namespace {

constexpr int kIn = 252, kH = 64, kOut = 9;
constexpr int oW1 = 0, oB1 = oW1 + kIn * kH, oW2 = oB1 + kH, oB2 = oW2 + kH * kH, oW3 = oB2 + kH,
              oB3 = oW3 + kH * kOut, kParams = oB3 + kOut;
static_assert(kParams == 20937, "MLP parameter count");

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
    return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

// Strip band of computed coordinate c along an axis of nc cells: depth
// 1..w into the strip and side -1 / +1, or 0 / 0 off the band.
__device__ __forceinline__ void band_of(int c, int nc, int w, float &depth, float &side) {
    if (c < w) { depth = (float)(w - c) / (float)w; side = -1.0f; }
    else if (c >= nc - w) { depth = (float)(c - (nc - w) + 1) / (float)w; side = 1.0f; }
    else { depth = 0.0f; side = 0.0f; }
}

// Per-cell sums of squares of the velocities and of the stresses, and the
// RMS scale s of a neighbourhood from their sums over its 27 cells (two
// partial sums each, neighbours 0..13 and 14..26, added at the end): the
// velocities enter times rho*vp, s = sqrt((zimp^2 SV + SS) / 243).  The same
// operations, in the same order, in the training inputs and the inference
// kernel, so both see the same s.
__device__ __forceinline__ float sq_velocity(const float (&f)[9]) {
    return fmaf(f[2], f[2], fmaf(f[1], f[1], f[0] * f[0]));
}
__device__ __forceinline__ float sq_stress(const float (&f)[9]) {
    return fmaf(f[8], f[8], fmaf(f[7], f[7], fmaf(f[6], f[6], fmaf(f[5], f[5], fmaf(f[4], f[4], f[3] * f[3])))));
}
__device__ __forceinline__ float rms_scale(float sv, float ss, float zimp) {
    return sqrtf(fmaf(zimp * zimp, sv, ss) * (1.0f / 243.0f));
}

// The 252 inputs of computed cell (cx, cy, cz), passed one by one to emit(i,
// value); returns the RMS scale s and sets zimp = rho * vp.
template <class F>
__device__ __forceinline__ float strip_inputs(const Model &m, int w, int cx, int cy, int cz, float &zimp, F emit) {
    const int64_t c = pidx(m, cx + kHalo, cy + kHalo, cz + kHalo);
    const float b = m.b[c], lam = m.lam[c], mu = m.mu[c];
    const float rho = 1.0f / b, vp = sqrtf((lam + 2.0f * mu) * b), vs = sqrtf(mu * b);
    zimp = rho * vp;
    float sv[2] = {0.0f, 0.0f}, ss[2] = {0.0f, 0.0f};
    for (int n = 0; n < 27; ++n) {
        const int64_t o = c + (n % 3 - 1) + (int64_t)((n / 3) % 3 - 1) * m.px + (int64_t)(n / 9 - 1) * m.plane;
        float f[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) f[k] = m.f[k][o];
        sv[n >= 14] += sq_velocity(f);
        ss[n >= 14] += sq_stress(f);
    }
    const float s = rms_scale(sv[0] + sv[1], ss[0] + ss[1], zimp);
    const float inv = s > 0.0f ? 1.0f / s : 0.0f, zinv = zimp * inv;
    for (int n = 0; n < 27; ++n) {
        const int64_t o = c + (n % 3 - 1) + (int64_t)((n / 3) % 3 - 1) * m.px + (int64_t)(n / 9 - 1) * m.plane;
#pragma unroll
        for (int k = 0; k < 9; ++k) emit(n * 9 + k, m.f[k][o] * (k < 3 ? zinv : inv));
    }
    emit(243, vp * (1.0f / 3000.0f));
    emit(244, vs * (1.0f / 1732.0f));
    emit(245, rho * (1.0f / 2000.0f));
    float d, sd;
    band_of(cx, m.nxc, w, d, sd); emit(246, d); emit(249, sd);
    band_of(cy, m.nyc, w, d, sd); emit(247, d); emit(250, sd);
    band_of(cz, m.nzc, w, d, sd); emit(248, d); emit(251, sd);
    return s;
}

// Inputs of listed cells (training data).
__global__ void k_strip_features(Model m, int w, const int4 *cells, int n, float *X, float *scale, float *zimp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 q = cells[i];
    float z;
    const float s = strip_inputs(m, w, q.x, q.y, q.z, z, [&](int f, float v) { X[(int64_t)i * kIn + f] = v; });
    scale[i] = s;
    zimp[i] = z;
}

// Training-data support.  dst's 9 fields (whole GRID) from the window of
// src whose GRID origin is (x0, y0, z0), dst's 5-cell frame set to zero.
__global__ void k_copy_window(Model dst, Model src, int x0, int y0, int z0) {
    const int64_t n = (int64_t)dst.nx * dst.ny * dst.nz;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % dst.nx), y = (int)((i / dst.nx) % dst.ny), z = (int)(i / ((int64_t)dst.nx * dst.ny));
        const bool frame = x < kHalo || y < kHalo || z < kHalo || x >= dst.nx - kHalo || y >= dst.ny - kHalo ||
                           z >= dst.nz - kHalo;
        const int64_t di = pidx(dst, x, y, z), si = pidx(src, x + x0, y + y0, z + z0);
#pragma unroll
        for (int k = 0; k < 9; ++k) dst.f[k][di] = frame ? 0.0f : src.f[k][si];
    }
}

// The 9 fields of listed computed cells: out[i][k].
__global__ void k_sample_fields(Model m, const int4 *cells, int n, float *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 q = cells[i];
    const int64_t c = pidx(m, q.x + kHalo, q.y + kHalo, q.z + kHalo);
#pragma unroll
    for (int k = 0; k < 9; ++k) out[(int64_t)i * 9 + k] = m.f[k][c];
}

// ---- tensor-core inference --------------------------------------------------

constexpr int kRows = kStripRows;          // cells per tile = MMA M
constexpr int kK1 = 256;                   // layer-1 K: the 252 inputs and 4 zeros
constexpr int kN3 = 16;                    // layer-3 N: the 9 outputs and 7 zeros
constexpr int kStage = kStripStage;        // staged cells per box, (32+2)(2+2)(2+2) at most
// Weight image (bytes): W1, W2, W3 transposed to N x K, FP16, in the K-major
// core-matrix order of kmaj, then the biases b1, b2, b3 (b3 padded to 16) in FP32.
constexpr int kImgW1 = 0, kImgW2 = kImgW1 + kH * kK1 * 2, kImgW3 = kImgW2 + kH * kH * 2,
              kImgB = kImgW3 + kN3 * kH * 2, kImg = kImgB + (2 * kH + kN3) * 4;
constexpr int kImgPad = (kImg + 1023) / 1024 * 1024;
constexpr int kKHalf = kK1 / 2;                              // layer 1 runs in two halves of K
constexpr int kAOp = kRows * kKHalf * 2;                     // A operand of one group (one half of K)
constexpr int kStg = 11 * kStage * 4;                        // staged fields and sums of squares of one warpgroup
constexpr int kRed = 4 * kRows * 4;                          // partial sums of squares of one warpgroup
constexpr int kMed = 3 * kRows * 4;                          // b, lambda, mu of the next tile's cells
constexpr int kWgBytes = kAOp + (kStg + 1023) / 1024 * 1024 + kRed + kMed;
constexpr int kGroups = 3;                                   // tile groups per CTA
constexpr int kTcSmem = 128 + kImgPad + kGroups * kWgBytes + 64;   // + alignment, barriers, TMEM address
constexpr int kTcThreads = kGroups * 2 * kRows;              // groups of 256 threads: two threads per row
static_assert(kImg % 16 == 0, "weight image is copied in 16-byte pieces");
static_assert(kTcSmem <= 232448, "shared memory of one CTA");
constexpr uint32_t kTmemCols = 512;                          // 128 per group: D1/D3 at +0, D2 at +64

// Byte offset of element (row, k) of a K-major operand with KT columns: 8x8
// core matrices of 128 contiguous bytes (8 rows of 16 bytes), the K-adjacent
// core matrices 128 bytes apart (LBO), the next 8 rows KT*16 bytes on (SBO).
__host__ __device__ constexpr uint32_t kmaj(int row, int k, int KT) {
    return (uint32_t)((row >> 3) * (KT * 16) + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// Shared-memory matrix descriptor: start address, LBO 128 B, SBO KT*16 B,
// descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, int KT) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)((KT * 16) >> 4) << 32) |
           (1ull << 46);
}
// Instruction descriptor of kind::f16: FP32 accumulator, A and B FP16 and
// K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t instr_desc(int n) {
    return (1u << 4) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kRows >> 4) << 24);
}

__device__ __forceinline__ uint32_t saddr_of(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init1(uint64_t *bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr_of(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Bounded wait for the phase of the given parity: false after about 2 s.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity) {
    for (int i = 0; i < 2000; ++i) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, 1000000;\n"
            " selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok) : "r"(saddr_of(bar)), "r"(parity) : "memory");
        if (ok) return true;
    }
    return false;
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Barrier of one 256-thread warpgroup pair (named barrier 1 + g) that also
// ORs a flag over it.
__device__ __forceinline__ bool wg_sync_or(int g, bool flag) {
    uint32_t r;
    asm volatile(
        "{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.or.pred q, %2, 256, p;\n selp.u32 %0, 1, 0, q;\n}\n"
        : "=r"(r) : "r"((uint32_t)flag), "r"(g + 1) : "memory");
    return r != 0;
}
__device__ __forceinline__ void wg_sync(int g) { asm volatile("bar.sync %0, 256;" ::"r"(g + 1) : "memory"); }

// D[tmem] (+)= A[a] * B[b]^T over nk steps of K = 16 (M = 128, N = n); A and
// B are K-major with kta and ktb columns; acc: add to D from the first step.
__device__ __forceinline__ void mma_k(uint32_t tmem_d, uint32_t a, int kta, uint32_t b, int ktb, int nk, int n,
                                      bool acc) {
    const uint32_t id = instr_desc(n);
    for (int kk = 0; kk < nk; ++kk) {
        const uint64_t ad = smem_desc(a + kk * 256, kta), bd = smem_desc(b + kk * 256, ktb);
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.u32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
            ::"r"(tmem_d), "l"(ad), "l"(bd), "r"(id), "r"((uint32_t)(acc || kk > 0)) : "memory");
    }
}
__device__ __forceinline__ void mma_chain(uint32_t tmem_d, uint32_t a, uint32_t b, int KT, int n) {
    mma_k(tmem_d, a, KT, b, KT, KT / 16, n, false);
}
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr_of(bar))
                 : "memory");
}
// 16 consecutive FP32 columns of this thread's TMEM lane; the wait is inside
// the same statement so no use of the registers can move above it.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n"
        "tcgen05.wait::ld.sync.aligned;\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr) : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ uint32_t pack_half2(float a, float b) {
    const __half2 h = __floats2half2_rn(a, b);
    return *reinterpret_cast<const uint32_t *>(&h);
}
__device__ __forceinline__ void store_chunk(unsigned char *p, const float (&v)[8]) {
    *reinterpret_cast<uint4 *>(p) = make_uint4(pack_half2(v[0], v[1]), pack_half2(v[2], v[3]),
                                               pack_half2(v[4], v[5]), pack_half2(v[6], v[7]));
}

__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float ex2_approx(float x) {
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
// GELU(x) = x Phi(x) = max(x, 0) - |x| erfc(|x| / sqrt 2) / 2 for either sign
// of x, with erfc from the Chebyshev fit of Numerical Recipes (Press et al.,
// 2nd ed., section 6.2, erfcc): erfc(z) = t exp(P(t) - z^2), t = 1 / (1 + z / 2),
// P of degree 9, fractional error below 1.2e-7 for every z, the small
// negative tail included -- far below the half ulp of the binary16 the
// activation is stored in (2.4e-4 relative).  The factor 1/2 and the change
// to base 2 are folded into P's coefficients: erfc(z) / 2 =
// t 2^(P2(t) - x^2 log2(e) / 2) with P2 = (P - ln 2) log2(e).  Two values at a
// time with packed FP32x2 arithmetic; the reciprocal and 2^q on the SFU.
__device__ __forceinline__ float2 f2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 gelu_fast2(float2 x) {
    const float2 nax = make_float2(-fabsf(x.x), -fabsf(x.y));
    const float2 d = __ffma2_rn(nax, f2(-0.35355339f), f2(1.0f));
    const float2 t = make_float2(rcp_approx(d.x), rcp_approx(d.y));
    float2 p = __ffma2_rn(t, f2(0.2465172979f), f2(-1.186114945f));
    p = __ffma2_rn(t, p, f2(2.147474464f));
    p = __ffma2_rn(t, p, f2(-1.637753152f));
    p = __ffma2_rn(t, p, f2(0.4023215817f));
    p = __ffma2_rn(t, p, f2(-0.2687568603f));
    p = __ffma2_rn(t, p, f2(0.1396300565f));
    p = __ffma2_rn(t, p, f2(0.5397006155f));
    p = __ffma2_rn(t, p, f2(1.442729204f));
    p = __ffma2_rn(t, p, f2(-2.825748218f));
    const float2 q = __ffma2_rn(__fmul2_rn(x, f2(-0.72134752f)), x, p);
    const float2 e = make_float2(ex2_approx(q.x), ex2_approx(q.y));
    return __ffma2_rn(__fmul2_rn(nax, t), e, make_float2(fmaxf(x.x, 0.0f), fmaxf(x.y, 0.0f)));
}

// Hidden layer, columns c0 .. c0+31 of this thread's row: accumulators + bias,
// GELU, FP16 into row t of the next A operand (K = 64).
__device__ __forceinline__ void hidden_half(uint32_t taddr, const float *bias, unsigned char *a_op, int t, int c0) {
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        float v[16];
        tmem_ld16(taddr + c0 + c * 16, v);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            float g[8];
#pragma unroll
            for (int q = 0; q < 8; q += 2) {
                const float2 r = gelu_fast2(__fadd2_rn(make_float2(v[8 * h + q], v[8 * h + q + 1]),
                                                       make_float2(bias[c0 + 16 * c + 8 * h + q],
                                                                   bias[c0 + 16 * c + 8 * h + q + 1])));
                g[q] = r.x;
                g[q + 1] = r.y;
            }
            store_chunk(a_op + kmaj(t, c0 + 16 * c + 8 * h, kH), g);
        }
    }
}

// Weight image from the FP32 parameters (once per sgfd_set_learned_strip).
__global__ void k_weight_image(const float *p, unsigned char *img) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kH * kK1; i += gridDim.x * blockDim.x) {
        const int j = i / kK1, k = i % kK1;   // output j, input k
        *reinterpret_cast<__half *>(img + kImgW1 + kmaj(j, k, kK1)) =
            __float2half_rn(k < kIn ? p[oW1 + k * kH + j] : 0.0f);
        if (k < kH) {
            *reinterpret_cast<__half *>(img + kImgW2 + kmaj(j, k, kH)) = __float2half_rn(p[oW2 + k * kH + j]);
            if (j < kN3)
                *reinterpret_cast<__half *>(img + kImgW3 + kmaj(j, k, kH)) =
                    __float2half_rn(j < kOut ? p[oW3 + k * kOut + j] : 0.0f);
        }
        if (i < kH) {
            float *bias = reinterpret_cast<float *>(img + kImgB);
            bias[i] = p[oB1 + i];
            bias[kH + i] = p[oB2 + i];
            if (i < kN3) bias[2 * kH + i] = i < kOut ? p[oB3 + i] : 0.0f;
        }
    }
}

// Strip box of tile `td`: origin (computed coordinates) and extents.
struct Box {
    int x, y, z, ex, ey, ez;
};
__device__ __forceinline__ Box box_of(int4 td) { return {td.x, td.y, td.z, td.w & 255, (td.w >> 8) & 255, (td.w >> 16) & 255}; }

__device__ __forceinline__ void cp_async4(float *dst, const float *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(saddr_of(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Starts the asynchronous copies of tile td's box with its one-cell halo (the
// 9 fields, all 256 threads of a group) and of the medium of its cells
// (thread u for row u) into the group's staging area; cp_async_wait_all
// completes them.  Staged cell r = lx + ly sx + lz sxy; the quotients through
// a float reciprocal, exact here: (r + 1/2) / d stays 1/(2d) > 9e-4 away from
// an integer and the product errs by < 2e-4 for r < 544.
__device__ __forceinline__ void stage_async(const Model &m, int4 td, float *stg, float *med, int u) {
    const Box bx = box_of(td);
    const int sx = bx.ex + 2, sxy = sx * (bx.ey + 2), ns = sxy * (bx.ez + 2);
    const float inv_sx = 1.0f / (float)sx, inv_sxy = 1.0f / (float)sxy;
    for (int r = u; r < ns; r += 2 * kRows) {
        const int lz = __float2int_rz(((float)r + 0.5f) * inv_sxy), rr = r - lz * sxy;
        const int ly = __float2int_rz(((float)rr + 0.5f) * inv_sx), lx = rr - ly * sx;
        const int64_t gi = pidx(m, bx.x - 1 + lx + kHalo, bx.y - 1 + ly + kHalo, bx.z - 1 + lz + kHalo);
#pragma unroll
        for (int k = 0; k < 9; ++k) cp_async4(stg + k * kStage + r, m.f[k] + gi);
    }
    if (u < bx.ex * bx.ey * bx.ez) {
        const int lx = u % bx.ex, ly = (u / bx.ex) % bx.ey, lz = u / (bx.ex * bx.ey);
        const int64_t gc = pidx(m, bx.x + lx + kHalo, bx.y + ly + kHalo, bx.z + lz + kHalo);
        cp_async4(med + u, m.b + gc);
        cp_async4(med + kRows + u, m.lam + gc);
        cp_async4(med + 2 * kRows + u, m.mu + gc);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

// Sums over the neighbours N0 .. N1-1 of staged cell c0 of the staged
// per-cell sums of squares: velocities (sv) and stresses (ss).
template <int N0, int N1>
__device__ __forceinline__ void staged_sums(const float *stg, int c0, int sx, int sxy, float &sv, float &ss) {
    sv = 0.0f;
    ss = 0.0f;
#pragma unroll
    for (int n = N0; n < N1; ++n) {
        const int o = c0 + (n % 3 - 1) + ((n / 3) % 3 - 1) * sx + (n / 9 - 1) * sxy;
        sv += stg[9 * kStage + o];
        ss += stg[10 * kStage + o];
    }
}

// Inputs J0*8 .. J0*8+63 of row t (8 chunks of 8) from the staged fields,
// into columns col0 .. col0+63 of the half-K A operand.
template <int J0>
__device__ __forceinline__ void staged_inputs(const float *stg, int c0, int sx, int sxy, float zinv, float inv,
                                              const float (&ext)[9], unsigned char *a_op, int t, int col0) {
#pragma unroll
    for (int j = J0; j < J0 + 8; ++j) {
        float v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int f = 8 * j + q;
            if (f < 243) {
                const int n = f / 9, k = f % 9;
                const int o = c0 + (n % 3 - 1) + ((n / 3) % 3 - 1) * sx + (n / 9 - 1) * sxy;
                v[q] = stg[k * kStage + o] * (k < 3 ? zinv : inv);
            } else {
                v[q] = f < kIn ? ext[f - 243] : 0.0f;
            }
        }
        store_chunk(a_op + kmaj(t, col0 + 8 * (j - J0), kKHalf), v);
    }
}

// Network of every strip cell (ROWS = false), or of n input rows X (ROWS =
// true: the tensor-core path checked on given inputs, raw outputs to out).
// One CTA per SM with 768 threads in three groups of 256; group g takes tiles
// 3*blockIdx.x + g, then every 3*gridDim.x-th.  In a group, threads t and
// t + 128 (warps w and w + 4, which reach the same TMEM lanes) share row t of
// a tile: half h = 0 takes neighbours 0..13, inputs 0..127 and hidden
// columns 0..31, half h = 1 neighbours 14..26, inputs 128..255 (with the 9
// cell inputs) and hidden columns 32..63; half 0 runs the epilogue.
// delta[tile][k][128] receives the corrected fields f + a d (a d the energy-limited correction).
template <bool ROWS>
__global__ void __launch_bounds__(kTcThreads, 1)
k_strip_tc(Model m, int w, const int4 *tiles, int ntiles, const unsigned char *wimg, float *delta, const float *X,
           int64_t nrows, float *out, int *err) {
    extern __shared__ unsigned char smem_raw[];
    unsigned char *sm = smem_raw + ((128 - (saddr_of(smem_raw) & 127)) & 127);
    const int tid = threadIdx.x, g = tid >> 8, u = tid & 255, h = u >> 7, t = u & 127, warp = tid >> 5;
    unsigned char *a_op = sm + kImgPad + g * kWgBytes;
    float *stg = reinterpret_cast<float *>(a_op + kAOp);
    float *red = reinterpret_cast<float *>(a_op + kWgBytes - kRed - kMed);
    float *med = reinterpret_cast<float *>(a_op + kWgBytes - kMed);
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + kImgPad + kGroups * kWgBytes);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bar + kGroups);

    for (int i = tid; i < kImg / 16; i += blockDim.x)
        reinterpret_cast<uint4 *>(sm)[i] = reinterpret_cast<const uint4 *>(wimg)[i];
    if (tid < kGroups) mbar_init1(&bar[tid]);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr_of(tmem_slot)),
                     "r"(kTmemCols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_async_smem();   // the weight image is read by the tensor cores
    tc_before();
    __syncthreads();
    tc_after();
    const uint32_t tmem_base = *tmem_slot;
    const uint32_t tmem_g = tmem_base + (uint32_t)(g * 128);
    const uint32_t tmem = tmem_g + ((uint32_t)((warp & 3) * 32) << 16);
    const uint32_t a_s = saddr_of(a_op), w1_s = saddr_of(sm + kImgW1), w2_s = saddr_of(sm + kImgW2),
                   w3_s = saddr_of(sm + kImgW3);
    const float *b1 = reinterpret_cast<const float *>(sm + kImgB), *b2 = b1 + kH, *b3 = b2 + kH;
    uint64_t *mybar = &bar[g];
    uint32_t parity = 0;
    bool failed = false;

    const int nt = ROWS ? (int)((nrows + kRows - 1) / kRows) : ntiles;
    const int first = kGroups * (int)blockIdx.x + g, stride = kGroups * (int)gridDim.x;
    if (!ROWS && first < nt) stage_async(m, tiles[first], stg, med, u);
    for (int tile = first; tile < nt; tile += stride) {
        // ---- row t's set-up: scale s, cell medium ----
        float s = 0.0f, zimp = 1.0f, inv = 0.0f, zinv = 0.0f, rho = 0.0f, vp = 0.0f, fc[kOut];
        float c_b = 1.0f, c_lam = 0.0f, c_mu = 1.0f;
        int count, c0 = 0, cx = 0, cy = 0, cz = 0, sx = 0, sxy = 0;
        if (ROWS) {
            const int64_t first_row = (int64_t)tile * kRows;
            count = (int)(nrows - first_row < kRows ? nrows - first_row : kRows);
        } else {
            const Box bx = box_of(tiles[tile]);
            sx = bx.ex + 2;
            sxy = sx * (bx.ey + 2);
            const int ns = sxy * (bx.ez + 2);
            cp_async_wait_all();   // this tile's copies, started during the previous tile
            for (int r = u; r < ns; r += 2 * kRows) {
                float f[9];
#pragma unroll
                for (int k = 0; k < 9; ++k) f[k] = stg[k * kStage + r];
                stg[9 * kStage + r] = sq_velocity(f);
                stg[10 * kStage + r] = sq_stress(f);
            }
            wg_sync(g);
            count = bx.ex * bx.ey * bx.ez;
            if (t < count) {
                const int lx = t % bx.ex, ly = (t / bx.ex) % bx.ey, lz = t / (bx.ex * bx.ey);
                cx = bx.x + lx;
                cy = bx.y + ly;
                cz = bx.z + lz;
                c0 = (lx + 1) + (ly + 1) * sx + (lz + 1) * sxy;
                c_b = med[t];
                c_lam = med[kRows + t];
                c_mu = med[2 * kRows + t];
                rho = 1.0f / c_b;
                vp = sqrtf((c_lam + 2.0f * c_mu) * c_b);
                zimp = rho * vp;
                float sv, ss;
                if (h == 0) staged_sums<0, 14>(stg, c0, sx, sxy, sv, ss);
                else staged_sums<14, 27>(stg, c0, sx, sxy, sv, ss);
                red[(2 * h) * kRows + t] = sv;
                red[(2 * h + 1) * kRows + t] = ss;
            }
            wg_sync(g);
            if (t < count) {
                s = rms_scale(red[t] + red[2 * kRows + t], red[kRows + t] + red[3 * kRows + t], zimp);
                inv = s > 0.0f ? 1.0f / s : 0.0f;
                zinv = zimp * inv;
                if (h == 0) {
#pragma unroll
                    for (int k = 0; k < kOut; ++k) fc[k] = stg[k * kStage + c0];
                }
            }
        }

        // ---- layer 1 in two halves of K: D1 = A W1^T, the A operand holding
        // inputs 128*half .. 128*half+127 (row t: 64 of them per thread) ----
        bool bad = false;
        for (int half = 0; half < 2; ++half) {
            if (ROWS) {
                const float *x = X + ((int64_t)tile * kRows + t) * kIn;
#pragma unroll 2
                for (int j = 0; j < 8; ++j) {
                    const int k0 = kKHalf * half + 64 * h + 8 * j;
                    float v[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) v[q] = (t < count && k0 + q < kIn) ? x[k0 + q] : 0.0f;
                    store_chunk(a_op + kmaj(t, 64 * h + 8 * j, kKHalf), v);
                }
            } else if (t < count) {
                const float none[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};   // inputs 0..191 hold no cell inputs
                if (half == 0) {
                    if (h == 0) staged_inputs<0>(stg, c0, sx, sxy, zinv, inv, none, a_op, t, 0);
                    else staged_inputs<8>(stg, c0, sx, sxy, zinv, inv, none, a_op, t, 64);
                } else if (h == 0) {
                    staged_inputs<16>(stg, c0, sx, sxy, zinv, inv, none, a_op, t, 0);
                } else {
                    // the 9 cell inputs (243..251) are in this quarter only
                    float ext[9];
                    ext[0] = vp * (1.0f / 3000.0f);
                    ext[1] = sqrtf(c_mu * c_b) * (1.0f / 1732.0f);
                    ext[2] = rho * (1.0f / 2000.0f);
                    band_of(cx, m.nxc, w, ext[3], ext[6]);
                    band_of(cy, m.nyc, w, ext[4], ext[7]);
                    band_of(cz, m.nzc, w, ext[5], ext[8]);
                    staged_inputs<24>(stg, c0, sx, sxy, zinv, inv, ext, a_op, t, 64);
                }
            } else {
                const float zero[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll 2
                for (int j = 0; j < 8; ++j) store_chunk(a_op + kmaj(t, 64 * h + 8 * j, kKHalf), zero);
            }
            fence_async_smem();
            tc_before();
            wg_sync(g);
            if (u == 0) {
                tc_after();
                mma_k(tmem_g, a_s, kKHalf, w1_s + half * (kKHalf / 16) * 256, kK1, kKHalf / 16, kH, half > 0);
                mma_commit(mybar);
            }
            // after the second half the staging area is free: the next tile's
            // copies overlap this one's network
            if (!ROWS && half == 1 && tile + stride < nt) stage_async(m, tiles[tile + stride], stg, med, u);
            const bool ok = mbar_wait_bounded(mybar, parity);
            parity ^= 1u;
            bad = wg_sync_or(g, !ok);
            if (bad) break;
            tc_after();
        }
        if (bad) { failed = true; break; }
        hidden_half(tmem, b1, a_op, t, 32 * h);

        // ---- layer 2: D2 = H1 (128 x 64) W2^T ----
        fence_async_smem();
        tc_before();
        wg_sync(g);
        if (u == 0) {
            tc_after();
            mma_chain(tmem_g + 64, a_s, w2_s, kH, kH);
            mma_commit(mybar);
        }
        bool ok = mbar_wait_bounded(mybar, parity);
        parity ^= 1u;
        if (wg_sync_or(g, !ok)) { failed = true; break; }
        tc_after();
        hidden_half(tmem + 64, b2, a_op, t, 32 * h);

        // ---- layer 3: D3 = H2 (128 x 64) W3^T, N = 16 ----
        fence_async_smem();
        tc_before();
        wg_sync(g);
        if (u == 0) {
            tc_after();
            mma_chain(tmem_g, a_s, w3_s, kH, kN3);
            mma_commit(mybar);
        }
        ok = mbar_wait_bounded(mybar, parity);
        parity ^= 1u;
        if (wg_sync_or(g, !ok)) { failed = true; break; }
        tc_after();

        // ---- epilogue (half 0) ----
        if (h == 0) {
            float o16[16];
            tmem_ld16(tmem, o16);
            if (t < count) {
                if (ROWS) {
                    const int64_t row = (int64_t)tile * kRows + t;
#pragma unroll
                    for (int k = 0; k < kOut; ++k) out[row * kOut + k] = o16[k] + b3[k];
                } else {
                    // Energy limit: the correction d may not raise the cell's energy
                    // E(f) = rho/2 |v|^2 + (s:s - c tr(s)^2) / (4 mu), c = lambda / (3 lambda + 2 mu)
                    // (the energy audit's density).  E(f + a d) = E(f) + 2 a B + a^2 Q, so the
                    // largest admissible a in [0, 1] is -2B/Q when B < 0, else 0.  A network
                    // trained on one-step targets is otherwise free to feed energy back into
                    // the strip and grow over long runs.
                    float d[kOut];
#pragma unroll
                    for (int k = 0; k < kOut; ++k) d[k] = (o16[k] + b3[k]) * s / (k < 3 ? zimp : 1.0f);
                    const float rho = 1.0f / c_b, lam = c_lam, mu = c_mu;
                    const float cc = lam / (3.0f * lam + 2.0f * mu), i4m = 0.25f / mu;
                    const float trf = fc[3] + fc[4] + fc[5], trd = d[3] + d[4] + d[5];
                    const float B = 0.5f * rho * (fc[0] * d[0] + fc[1] * d[1] + fc[2] * d[2]) +
                                    i4m * (fc[3] * d[3] + fc[4] * d[4] + fc[5] * d[5] +
                                           2.0f * (fc[6] * d[6] + fc[7] * d[7] + fc[8] * d[8]) - cc * trf * trd);
                    const float Q = 0.5f * rho * (d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) +
                                    i4m * (d[3] * d[3] + d[4] * d[4] + d[5] * d[5] +
                                           2.0f * (d[6] * d[6] + d[7] * d[7] + d[8] * d[8]) - cc * trd * trd);
                    const float a = (Q > 0.0f && B < 0.0f) ? fminf(1.0f, -2.0f * B / Q) : 0.0f;
                    float *dt = delta + (int64_t)tile * (kRows * kOut);
#pragma unroll
                    for (int k = 0; k < kOut; ++k) dt[k * kRows + t] = fc[k] + a * d[k];
                }
            }
        }
    }
    cp_async_wait_all();
    if (failed) {
        if (u == 0) atomicOr(err, 4);
        mbar_wait_bounded(mybar, parity ^ 1u);   // the commit the failed wait was for
    }
    tc_before();
    __syncthreads();
    if (warp == 0) {
        tc_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(kTmemCols)
                     : "memory");
    }
}

// One CTA per SM (fewer for small strips): each runs kGroups tile groups.
int tc_grid(int ntiles) {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return std::max(1, std::min(sms, (ntiles + kGroups - 1) / kGroups));
}

// Writes the corrected fields into the strip cells (after every cell's
// correction has been computed from the uncorrected state).  One block per
// tile; k_strip_tc left f + a d for each cell in delta[tile][k][128].
__global__ void __launch_bounds__(kRows) k_strip_apply(Model m, const int4 *tiles, const float *delta) {
    const Box bx = box_of(tiles[blockIdx.x]);
    const int t = threadIdx.x;
    if (t >= bx.ex * bx.ey * bx.ez) return;
    const int lx = t % bx.ex, ly = (t / bx.ex) % bx.ey, lz = t / (bx.ex * bx.ey);
    const int64_t c = pidx(m, bx.x + lx + kHalo, bx.y + ly + kHalo, bx.z + lz + kHalo);
    const float *dt = delta + (int64_t)blockIdx.x * (kRows * kOut);
    float v[kOut];   // every load before the first store (the arrays could alias as far as the compiler knows)
#pragma unroll
    for (int k = 0; k < kOut; ++k) v[k] = dt[k * kRows + t];
#pragma unroll
    for (int k = 0; k < kOut; ++k) m.f[k][c] = v[k];
}

// ---- training kernels ------------------------------------------------------

// C[M][N] = op(A)[M][K] * op(B)[K][N] (+ C when acc), row-major; op = transpose
// when TA / TB (A stored [K][M], B stored [N][K]).  16x16 tiles.
template <bool TA, bool TB>
__global__ void k_gemm(int M, int N, int K, const float *A, const float *B, float *C, int acc) {
    __shared__ float As[16][17], Bs[16][17];
    const int r = blockIdx.y * 16 + threadIdx.y, cidx = blockIdx.x * 16 + threadIdx.x;
    float sum = 0.0f;
    for (int k0 = 0; k0 < K; k0 += 16) {
        const int ka = k0 + threadIdx.x, kb = k0 + threadIdx.y;
        const int ar = blockIdx.y * 16 + threadIdx.y, bc = blockIdx.x * 16 + threadIdx.x;
        As[threadIdx.y][threadIdx.x] = (ar < M && ka < K) ? (TA ? A[(int64_t)ka * M + ar] : A[(int64_t)ar * K + ka]) : 0.0f;
        Bs[threadIdx.y][threadIdx.x] = (kb < K && bc < N) ? (TB ? B[(int64_t)bc * K + kb] : B[(int64_t)kb * N + bc]) : 0.0f;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 16; ++k) sum = fmaf(As[threadIdx.y][k], Bs[k][threadIdx.x], sum);
        __syncthreads();
    }
    if (r < M && cidx < N) C[(int64_t)r * N + cidx] = acc ? C[(int64_t)r * N + cidx] + sum : sum;
}

// Z += bias (per column); A = GELU(Z).
__global__ void k_bias_gelu(float *Z, const float *bias, float *A, int M, int N) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (int64_t)M * N) return;
    const float z = Z[i] + bias[i % N];
    Z[i] = z;
    A[i] = gelu(z);
}

// Output layer: Z += b3; dZ = 2 (Z - Y) / (M * 9); loss += sum (Z - Y)^2 / (M * 9).
__global__ void k_out_loss(float *Z, const float *bias, const float *Y, float *dZ, int M, float *loss) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    float e2 = 0.0f;
    if (i < (int64_t)M * kOut) {
        const float z = Z[i] + bias[i % kOut];
        Z[i] = z;
        const float d = z - Y[i];
        dZ[i] = 2.0f * d / ((float)M * kOut);
        e2 = d * d / ((float)M * kOut);
    }
    for (int o = 16; o > 0; o >>= 1) e2 += __shfl_xor_sync(0xffffffffu, e2, o);
    if ((threadIdx.x & 31) == 0 && loss) atomicAdd(loss, e2);
}

__global__ void k_gelu_back(float *dA, const float *Z, int64_t count) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < count) dA[i] *= gelu_grad(Z[i]);
}

__global__ void k_colsum(const float *D, int M, int N, float *out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= N) return;
    float s = 0.0f;
    for (int i = 0; i < M; ++i) s += D[(int64_t)i * N + j];
    out[j] = s;
}

__global__ void k_adam(float *p, const float *g, float *m1, float *m2, int n, float lr, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    m1[i] = 0.9f * m1[i] + 0.1f * gi;
    m2[i] = 0.999f * m2[i] + 0.001f * gi * gi;
    p[i] -= lr * (m1[i] / c1) / (sqrtf(m2[i] / c2) + 1e-8f);
}

inline unsigned cdiv(int64_t a, int64_t b) { return (unsigned)((a + b - 1) / b); }

template <bool TA, bool TB>
void gemm(int M, int N, int K, const float *A, const float *B, float *C, bool acc, cudaStream_t s) {
    k_gemm<TA, TB><<<dim3(cdiv(N, 16), cdiv(M, 16)), dim3(16, 16), 0, s>>>(M, N, K, A, B, C, acc ? 1 : 0);
}

// Device workspace of one minibatch of at most B samples.
struct Mlp {
    int B = 0;
    float *p = nullptr, *g = nullptr, *m1 = nullptr, *m2 = nullptr;
    float *Z1 = nullptr, *A1 = nullptr, *Z2 = nullptr, *A2 = nullptr, *Z3 = nullptr, *D3 = nullptr;
    float *loss = nullptr;
    cudaError_t alloc(int batch) {
        B = batch;
        const size_t a = (size_t)B * kH * sizeof(float);
        cudaError_t e = cudaMalloc(&p, 4 * (size_t)kParams * sizeof(float));
        if (e == cudaSuccess) e = cudaMalloc(&Z1, 4 * a + 2 * (size_t)B * kOut * sizeof(float) + sizeof(float));
        if (e != cudaSuccess) return e;
        g = p + kParams; m1 = g + kParams; m2 = m1 + kParams;
        A1 = Z1 + (size_t)B * kH; Z2 = A1 + (size_t)B * kH; A2 = Z2 + (size_t)B * kH;
        Z3 = A2 + (size_t)B * kH; D3 = Z3 + (size_t)B * kOut; loss = D3 + (size_t)B * kOut;
        return cudaMemset(m1, 0, 2 * (size_t)kParams * sizeof(float));
    }
    void release() { cudaFree(p); cudaFree(Z1); p = Z1 = nullptr; }

    void forward(const float *X, int n, cudaStream_t s) {
        gemm<false, false>(n, kH, kIn, X, p + oW1, Z1, false, s);
        k_bias_gelu<<<cdiv((int64_t)n * kH, 256), 256, 0, s>>>(Z1, p + oB1, A1, n, kH);
        gemm<false, false>(n, kH, kH, A1, p + oW2, Z2, false, s);
        k_bias_gelu<<<cdiv((int64_t)n * kH, 256), 256, 0, s>>>(Z2, p + oB2, A2, n, kH);
        gemm<false, false>(n, kOut, kH, A2, p + oW3, Z3, false, s);
    }
    // loss and gradient of one batch (after forward)
    void backward(const float *X, const float *Y, int n, cudaStream_t s) {
        k_out_loss<<<cdiv((int64_t)n * kOut, 256), 256, 0, s>>>(Z3, p + oB3, Y, D3, n, loss);
        gemm<true, false>(kH, kOut, n, A2, D3, g + oW3, false, s);        // dW3 = A2^T dZ3
        k_colsum<<<1, kOut, 0, s>>>(D3, n, kOut, g + oB3);
        gemm<false, true>(n, kH, kOut, D3, p + oW3, A2, false, s);        // dA2 = dZ3 W3^T (into A2)
        k_gelu_back<<<cdiv((int64_t)n * kH, 256), 256, 0, s>>>(A2, Z2, (int64_t)n * kH);
        gemm<true, false>(kH, kH, n, A1, A2, g + oW2, false, s);          // dW2 = A1^T dZ2
        k_colsum<<<1, kH, 0, s>>>(A2, n, kH, g + oB2);
        gemm<false, true>(n, kH, kH, A2, p + oW2, A1, false, s);          // dA1 = dZ2 W2^T (into A1)
        k_gelu_back<<<cdiv((int64_t)n * kH, 256), 256, 0, s>>>(A1, Z1, (int64_t)n * kH);
        gemm<true, false>(kIn, kH, n, X, A1, g + oW1, false, s);          // dW1 = X^T dZ1
        k_colsum<<<1, kH, 0, s>>>(A1, n, kH, g + oB1);
    }
};

int mlp_fail(const char *what, cudaError_t e) {
    return fail(nullptr, SGFD_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

}  // namespace

extern "C" {

int sgfd_mlp_param_count(void) { return kParams; }

int sgfd_mlp_forward(int32_t device, const float *params, const float *X, int64_t n, float *out) {
    if (!params || !X || !out || n <= 0) return fail(nullptr, SGFD_ERR_INVALID, "bad MLP forward arguments");
    cudaError_t e = cudaSetDevice(device);
    Mlp mlp;
    float *dX = nullptr;
    if (e == cudaSuccess) e = mlp.alloc((int)n);
    if (e == cudaSuccess) e = cudaMalloc(&dX, (size_t)n * kIn * sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpy(mlp.p, params, kParams * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dX, X, (size_t)n * kIn * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        mlp.forward(dX, (int)n, 0);
        e = cudaGetLastError();
    }
    // the output bias is added on the host
    std::vector<float> z((size_t)n * kOut), b3(kOut);
    if (e == cudaSuccess) e = cudaMemcpy(z.data(), mlp.Z3, z.size() * sizeof(float), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(b3.data(), mlp.p + oB3, kOut * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(dX);
    mlp.release();
    if (e != cudaSuccess) return mlp_fail("MLP forward", e);
    for (int64_t i = 0; i < n; ++i)
        for (int k = 0; k < kOut; ++k) out[i * kOut + k] = z[i * kOut + k] + b3[k];
    return SGFD_OK;
}

int sgfd_mlp_infer(int32_t device, const float *params, const float *X, int64_t n, float *out) {
    if (!params || !X || !out || n <= 0 || n > ((int64_t)1 << 30))
        return fail(nullptr, SGFD_ERR_INVALID, "bad MLP inference arguments");
    cudaError_t e = cudaSetDevice(device);
    unsigned char *img = nullptr;
    float *dp = nullptr, *dX = nullptr, *dout = nullptr;
    int *err = nullptr;
    const int nt = (int)((n + kRows - 1) / kRows);
    if (e == cudaSuccess) e = strip_prepare();
    if (e == cudaSuccess) e = cudaMalloc(&img, kImgPad + 16);
    if (e == cudaSuccess) e = cudaMalloc(&dp, kParams * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&dX, (size_t)n * kIn * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&dout, (size_t)n * kOut * sizeof(float));
    if (e == cudaSuccess) e = cudaMemset(img, 0, kImgPad + 16);
    if (e == cudaSuccess) e = cudaMemcpy(dp, params, kParams * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dX, X, (size_t)n * kIn * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        err = reinterpret_cast<int *>(img + kImgPad);
        k_weight_image<<<64, 256>>>(dp, img);
        k_strip_tc<true><<<tc_grid(nt), kTcThreads, kTcSmem>>>(Model{}, 0, nullptr, 0, img, nullptr, dX, n, dout, err);
        e = cudaGetLastError();
    }
    int flag = 0;
    if (e == cudaSuccess) e = cudaMemcpy(out, dout, (size_t)n * kOut * sizeof(float), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&flag, err, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(img);
    cudaFree(dp);
    cudaFree(dX);
    cudaFree(dout);
    if (e != cudaSuccess) return mlp_fail("MLP inference", e);
    if (flag) return fail(nullptr, SGFD_ERR_CUDA, "MLP inference: a bounded wait for tensor-core results gave up");
    return SGFD_OK;
}

int sgfd_mlp_gradient(int32_t device, const float *params, const float *X, const float *Y, int32_t n, float *loss,
                      float *grad) {
    if (!params || !X || !Y || !grad || n <= 0) return fail(nullptr, SGFD_ERR_INVALID, "bad MLP gradient arguments");
    cudaError_t e = cudaSetDevice(device);
    Mlp mlp;
    float *dX = nullptr, *dY = nullptr;
    if (e == cudaSuccess) e = mlp.alloc(n);
    if (e == cudaSuccess) e = cudaMalloc(&dX, (size_t)n * (kIn + kOut) * sizeof(float));
    if (e == cudaSuccess) {
        dY = dX + (size_t)n * kIn;
        e = cudaMemcpy(mlp.p, params, kParams * sizeof(float), cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) e = cudaMemcpy(dX, X, (size_t)n * kIn * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dY, Y, (size_t)n * kOut * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(mlp.loss, 0, sizeof(float));
    if (e == cudaSuccess) {
        mlp.forward(dX, n, 0);
        mlp.backward(dX, dY, n, 0);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(grad, mlp.g, kParams * sizeof(float), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && loss) e = cudaMemcpy(loss, mlp.loss, sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(dX);
    mlp.release();
    return e == cudaSuccess ? SGFD_OK : mlp_fail("MLP gradient", e);
}

int sgfd_mlp_train(int32_t device, float *params, const float *X, const float *Y, int64_t n, int32_t epochs,
                   int32_t batch, float lr, float *epoch_loss) {
    if (!params || !X || !Y || n <= 0 || epochs <= 0 || batch <= 0 || !(lr > 0))
        return fail(nullptr, SGFD_ERR_INVALID, "bad MLP training arguments");
    cudaError_t e = cudaSetDevice(device);
    Mlp mlp;
    float *dX = nullptr;
    const int B = (int)std::min<int64_t>(batch, n);
    if (e == cudaSuccess) e = mlp.alloc(B);
    if (e == cudaSuccess) e = cudaMalloc(&dX, (size_t)n * (kIn + kOut) * sizeof(float));
    float *dY = dX ? dX + (size_t)n * kIn : nullptr;
    if (e == cudaSuccess) e = cudaMemcpy(mlp.p, params, kParams * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dX, X, (size_t)n * kIn * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dY, Y, (size_t)n * kOut * sizeof(float), cudaMemcpyHostToDevice);
    int64_t t = 0;
    for (int ep = 0; ep < epochs && e == cudaSuccess; ++ep) {
        e = cudaMemset(mlp.loss, 0, sizeof(float));
        int nb = 0;
        for (int64_t b0 = 0; b0 + B <= n && e == cudaSuccess; b0 += B, ++nb) {
            mlp.forward(dX + b0 * kIn, B, 0);
            mlp.backward(dX + b0 * kIn, dY + b0 * kOut, B, 0);
            ++t;
            const float c1 = 1.0f - std::pow(0.9f, (float)t), c2 = 1.0f - std::pow(0.999f, (float)t);
            k_adam<<<cdiv(kParams, 256), 256>>>(mlp.p, mlp.g, mlp.m1, mlp.m2, kParams, lr, c1, c2);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess && epoch_loss) {
            float l = 0.0f;
            e = cudaMemcpy(&l, mlp.loss, sizeof(float), cudaMemcpyDeviceToHost);
            epoch_loss[ep] = nb ? l / (float)nb : 0.0f;
        }
    }
    if (e == cudaSuccess) e = cudaMemcpy(params, mlp.p, kParams * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(dX);
    mlp.release();
    return e == cudaSuccess ? SGFD_OK : mlp_fail("MLP training", e);
}

int sgfd_set_learned_strip(sgfd_solver *h, int32_t width, const float *params) {
    int r = check_handle(h);
    if (r) return r;
    if (width < 0) return fail(h, SGFD_ERR_INVALID, "negative strip width");
    if (width > 0 && h->cfg.nz_total != 0) return fail(h, SGFD_ERR_UNSUPPORTED, "a z-slab takes no learned strip");
    SG_CUDA(h, cudaStreamSynchronize(h->stream), "synchronise before changing the strip");
    cudaFree(h->strip_cells);
    cudaFree(h->strip_buf);
    h->strip_cells = nullptr;
    h->strip_buf = nullptr;
    h->strip_w = h->strip_n = 0;
    if (width == 0) return SGFD_OK;
    if (!params) return fail(h, SGFD_ERR_INVALID, "null strip parameters");
    if (h->cfg.pml != 0)
        return fail(h, SGFD_ERR_INVALID, "the learned strip replaces the PML: create the model with pml = 0");
    if (h->storage != SGFD_STORE_F32) return fail(h, SGFD_ERR_UNSUPPORTED, "the learned strip needs FP32 storage");
    const Model &m = h->m;
    if (2 * width >= std::min(m.nxc, std::min(m.nyc, m.nzc)))
        return fail(h, SGFD_ERR_INVALID, "strip width %d leaves no interior", width);
    std::vector<int4> tiles;
    const int nt = strip_tile_list(m, width, tiles);
    if (nt <= 0) return fail(h, SGFD_ERR_INVALID, "strip width %d: no strip tiling", width);
    SG_CUDA(h, strip_prepare(), "strip kernel set-up");
    SG_CUDA(h, dev_malloc(h, &h->strip_cells, (size_t)nt * sizeof(int4)), "strip tiles");
    SG_CUDA(h, dev_malloc(h, &h->strip_buf, strip_buffer_bytes(nt)), "strip buffers");
    SG_CUDA(h, cudaMemcpy(h->strip_cells, tiles.data(), (size_t)nt * sizeof(int4), cudaMemcpyHostToDevice), "strip tiles");
    SG_CUDA(h, cudaMemset(h->strip_buf, 0, strip_buffer_bytes(nt)), "strip buffers");
    float *dp = nullptr;
    SG_CUDA(h, dev_malloc(h, &dp, (size_t)kParams * sizeof(float)), "strip parameters");
    cudaError_t e = cudaMemcpy(dp, params, (size_t)kParams * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_weight_image<<<64, 256>>>(dp, reinterpret_cast<unsigned char *>(h->strip_buf));
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    cudaFree(dp);
    if (e != cudaSuccess) return cuda_fail(h, e, "strip weight image");
    h->strip_w = width;
    h->strip_n = nt;
    return SGFD_OK;
}

int sgfd_copy_window(sgfd_solver *dst, sgfd_solver *src, int32_t x0, int32_t y0, int32_t z0) {
    int r = check_handle(src);
    if (r) return r;
    r = check_handle(dst);
    if (r) return r;
    if (dst->device != src->device) return fail(dst, SGFD_ERR_INVALID, "the two models are on different devices");
    if (dst->cfg.pml != 0) return fail(dst, SGFD_ERR_INVALID, "the destination model must have pml = 0");
    if (dst->storage != SGFD_STORE_F32 || src->storage != SGFD_STORE_F32)
        return fail(dst, SGFD_ERR_UNSUPPORTED, "window copies need FP32 storage");
    const Model &d = dst->m, &s = src->m;
    if (x0 < 0 || y0 < 0 || z0 < 0 || x0 + d.nx > s.nx || y0 + d.ny > s.ny || z0 + d.nz > s.nz)
        return fail(dst, SGFD_ERR_INVALID, "window (%d,%d,%d)+(%d,%d,%d) outside the source grid", x0, y0, z0, d.nx,
                    d.ny, d.nz);
    // dst's stream waits for src's queued steps, src's for this copy
    cudaEvent_t ev = nullptr;
    SG_CUDA(dst, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "window event");
    cudaError_t e = cudaEventRecord(ev, src->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(dst->stream, ev, 0);
    if (e == cudaSuccess) {
        k_copy_window<<<1184, 256, 0, dst->stream>>>(d, s, x0, y0, z0);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventRecord(ev, dst->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(src->stream, ev, 0);
    cudaEventDestroy(ev);
    return e == cudaSuccess ? SGFD_OK : cuda_fail(dst, e, "window copy");
}

int sgfd_sample_fields(sgfd_solver *h, int32_t n, const int32_t *cells, float *out) {
    int r = check_handle(h);
    if (r) return r;
    if (n < 0 || (n && (!cells || !out))) return fail(h, SGFD_ERR_INVALID, "bad sample arguments");
    if (n == 0) return SGFD_OK;
    const Model &m = h->m;
    std::vector<int4> c(n);
    for (int i = 0; i < n; ++i) {
        c[i] = make_int4(cells[3 * i], cells[3 * i + 1], cells[3 * i + 2], 0);
        if (c[i].x < 0 || c[i].y < 0 || c[i].z < 0 || c[i].x >= m.nxc || c[i].y >= m.nyc || c[i].z >= m.nzc)
            return fail(h, SGFD_ERR_INVALID, "cell %d is outside the computed region", i);
    }
    r = sync_views(h);
    if (r) return r;
    int4 *dc = nullptr;
    float *dout = nullptr;
    SG_CUDA(h, dev_malloc(h, &dc, (size_t)n * sizeof(int4)), "sample scratch");
    cudaError_t e = dev_malloc(h, &dout, (size_t)n * 9 * sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpyAsync(dc, c.data(), (size_t)n * sizeof(int4), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) {
        k_sample_fields<<<cdiv(n, 128), 128, 0, h->stream>>>(m, dc, n, dout);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, dout, (size_t)n * 9 * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(dc);
    cudaFree(dout);
    return e == cudaSuccess ? SGFD_OK : cuda_fail(h, e, "field samples");
}

int sgfd_strip_features(sgfd_solver *h, int32_t width, int32_t n, const int32_t *cells, float *X, float *scale,
                        float *zimp) {
    int r = check_handle(h);
    if (r) return r;
    if (width < 1 || n < 0 || (n && (!cells || !X || !scale || !zimp)))
        return fail(h, SGFD_ERR_INVALID, "bad strip feature arguments");
    if (n == 0) return SGFD_OK;
    const Model &m = h->m;
    std::vector<int4> c(n);
    for (int i = 0; i < n; ++i) {
        c[i] = make_int4(cells[3 * i], cells[3 * i + 1], cells[3 * i + 2], 0);
        if (c[i].x < 0 || c[i].y < 0 || c[i].z < 0 || c[i].x >= m.nxc || c[i].y >= m.nyc || c[i].z >= m.nzc)
            return fail(h, SGFD_ERR_INVALID, "cell %d is outside the computed region", i);
    }
    r = sync_views(h);
    if (r) return r;
    int4 *dc = nullptr;
    float *dX = nullptr;
    SG_CUDA(h, dev_malloc(h, &dc, (size_t)n * sizeof(int4)), "feature scratch");
    cudaError_t e = dev_malloc(h, &dX, (size_t)n * (kIn + 2) * sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpyAsync(dc, c.data(), (size_t)n * sizeof(int4), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) {
        k_strip_features<<<cdiv(n, 128), 128, 0, h->stream>>>(m, width, dc, n, dX, dX + (size_t)n * kIn,
                                                              dX + (size_t)n * (kIn + 1));
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(X, dX, (size_t)n * kIn * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(scale, dX + (size_t)n * kIn, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(zimp, dX + (size_t)n * (kIn + 1), (size_t)n * sizeof(float), cudaMemcpyDeviceToHost,
                            h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(dc);
    cudaFree(dX);
    return e == cudaSuccess ? SGFD_OK : cuda_fail(h, e, "strip features");
}

}  // extern "C"

namespace sgfd {

// The strip's tiles (strip_tiles.h) for model m.
int strip_tile_list(const Model &m, int w, std::vector<int4> &tiles) { return strip_tiles(m.nxc, m.nyc, m.nzc, w, tiles); }

// Strip buffer: weight image, corrected fields [tile][9][128], error flag.
size_t strip_buffer_bytes(int ntiles) { return (size_t)kImgPad + (size_t)ntiles * kRows * kOut * 4 + 16; }
int *strip_error_flag(float *buf, int ntiles) {
    return reinterpret_cast<int *>(reinterpret_cast<unsigned char *>(buf) + strip_buffer_bytes(ntiles) - 16);
}

cudaError_t strip_prepare() {
    cudaError_t e = cudaFuncSetAttribute(k_strip_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_strip_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem);
    return e;
}

cudaError_t launch_strip(const Model &m, int w, const int4 *tiles, int ntiles, float *buf, cudaStream_t s) {
    const unsigned char *img = reinterpret_cast<const unsigned char *>(buf);
    float *delta = reinterpret_cast<float *>(reinterpret_cast<unsigned char *>(buf) + kImgPad);
    k_strip_tc<false><<<tc_grid(ntiles), kTcThreads, kTcSmem, s>>>(m, w, tiles, ntiles, img, delta, nullptr, 0, nullptr,
                                                            strip_error_flag(buf, ntiles));
    k_strip_apply<<<ntiles, kRows, 0, s>>>(m, tiles, delta);
    return cudaGetLastError();
}

int mlp_params() { return kParams; }

}  // namespace sgfd
