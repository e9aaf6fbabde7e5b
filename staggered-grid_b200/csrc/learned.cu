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
//     energy (k_strip_mlp).
// Parameters, 20 937 floats: W1 [252][64], b1, W2 [64][64], b2, W3 [64][9], b3.
//
// Training (sgfd_mlp_train) runs minibatch Adam with hand-written kernels:
// a tiled FP32 GEMM, bias + GELU, the output loss (mean squared error over the
// 9 outputs), the GELU backward, column sums and the Adam update.  The
// gradients are checked against a CPU restatement in the tests.
#include <cmath>
#include <cstring>
#include <vector>

#include "solver.h"

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

// The 252 inputs of computed cell (cx, cy, cz), passed one by one to emit(i,
// value); returns the RMS scale s and sets zimp = rho * vp.
template <class F>
__device__ __forceinline__ float strip_inputs(const Model &m, int w, int cx, int cy, int cz, float &zimp, F emit) {
    const int64_t c = pidx(m, cx + kHalo, cy + kHalo, cz + kHalo);
    const float b = m.b[c], lam = m.lam[c], mu = m.mu[c];
    const float rho = 1.0f / b, vp = sqrtf((lam + 2.0f * mu) * b), vs = sqrtf(mu * b);
    zimp = rho * vp;
    float ss = 0.0f;
    for (int n = 0; n < 27; ++n) {
        const int64_t o = c + (n % 3 - 1) + (int64_t)((n / 3) % 3 - 1) * m.px + (int64_t)(n / 9 - 1) * m.plane;
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            const float u = m.f[k][o] * (k < 3 ? zimp : 1.0f);
            ss = fmaf(u, u, ss);
        }
    }
    const float s = sqrtf(ss * (1.0f / 243.0f));
    const float inv = s > 0.0f ? 1.0f / s : 0.0f;
    for (int n = 0; n < 27; ++n) {
        const int64_t o = c + (n % 3 - 1) + (int64_t)((n / 3) % 3 - 1) * m.px + (int64_t)(n / 9 - 1) * m.plane;
#pragma unroll
        for (int k = 0; k < 9; ++k) emit(n * 9 + k, m.f[k][o] * (k < 3 ? zimp : 1.0f) * inv);
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

// Corrections of all strip cells from the current state (one thread per
// cell, the parameters in shared memory).  Written to delta first and added
// by k_strip_apply, so that every correction sees the uncorrected state.
__global__ void __launch_bounds__(128) k_strip_mlp(Model m, int w, const int4 *cells, int n, const float *params,
                                                   float *delta) {
    extern __shared__ float wsm[];
    for (int i = threadIdx.x; i < kParams; i += blockDim.x) wsm[i] = params[i];
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 q = cells[i];
    float h1[kH];
#pragma unroll
    for (int j = 0; j < kH; ++j) h1[j] = wsm[oB1 + j];
    float z;
    const float s = strip_inputs(m, w, q.x, q.y, q.z, z, [&](int f, float v) {
        const float *row = wsm + oW1 + f * kH;
#pragma unroll
        for (int j = 0; j < kH; ++j) h1[j] = fmaf(v, row[j], h1[j]);
    });
#pragma unroll
    for (int j = 0; j < kH; ++j) h1[j] = gelu(h1[j]);
    float out[kOut];
#pragma unroll
    for (int k = 0; k < kOut; ++k) out[k] = wsm[oB3 + k];
    for (int j2 = 0; j2 < kH; ++j2) {
        float a = wsm[oB2 + j2];
#pragma unroll
        for (int j = 0; j < kH; ++j) a = fmaf(h1[j], wsm[oW2 + j * kH + j2], a);
        a = gelu(a);
#pragma unroll
        for (int k = 0; k < kOut; ++k) out[k] = fmaf(a, wsm[oW3 + j2 * kOut + k], out[k]);
    }
    // Energy limit: the correction d may not raise the cell's energy
    // E(f) = rho/2 |v|^2 + (s:s - c tr(s)^2) / (4 mu), c = lambda / (3 lambda + 2 mu)
    // (the energy audit's density).  E(f + a d) = E(f) + 2 a B + a^2 Q, so the
    // largest admissible a in [0, 1] is -2B/Q when B < 0, else 0.  A network
    // trained on one-step targets is otherwise free to feed energy back into
    // the strip and grow over long runs.
    const int64_t c = pidx(m, q.x + kHalo, q.y + kHalo, q.z + kHalo);
    float f[kOut], d[kOut];
#pragma unroll
    for (int k = 0; k < kOut; ++k) {
        f[k] = m.f[k][c];
        d[k] = out[k] * s / (k < 3 ? z : 1.0f);
    }
    const float rho = 1.0f / m.b[c], lam = m.lam[c], mu = m.mu[c];
    const float cc = lam / (3.0f * lam + 2.0f * mu), i4m = 0.25f / mu;
    const float trf = f[3] + f[4] + f[5], trd = d[3] + d[4] + d[5];
    const float B = 0.5f * rho * (f[0] * d[0] + f[1] * d[1] + f[2] * d[2]) +
                    i4m * (f[3] * d[3] + f[4] * d[4] + f[5] * d[5] + 2.0f * (f[6] * d[6] + f[7] * d[7] + f[8] * d[8]) -
                           cc * trf * trd);
    const float Q = 0.5f * rho * (d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) +
                    i4m * (d[3] * d[3] + d[4] * d[4] + d[5] * d[5] + 2.0f * (d[6] * d[6] + d[7] * d[7] + d[8] * d[8]) -
                           cc * trd * trd);
    const float a = (Q > 0.0f && B < 0.0f) ? fminf(1.0f, -2.0f * B / Q) : 0.0f;
#pragma unroll
    for (int k = 0; k < kOut; ++k) delta[(int64_t)i * kOut + k] = a * d[k];
}

__global__ void k_strip_apply(Model m, const int4 *cells, int n, const float *delta) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 q = cells[i];
    const int64_t c = pidx(m, q.x + kHalo, q.y + kHalo, q.z + kHalo);
#pragma unroll
    for (int k = 0; k < kOut; ++k) m.f[k][c] += delta[(int64_t)i * kOut + k];
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
    std::vector<int4> cells;
    const int n = strip_cell_list(m, width, cells);
    SG_CUDA(h, strip_prepare(), "strip kernel set-up");
    SG_CUDA(h, cudaMalloc(&h->strip_cells, (size_t)n * sizeof(int4)), "strip cell list");
    SG_CUDA(h, cudaMalloc(&h->strip_buf, ((size_t)kParams + (size_t)n * kOut) * sizeof(float)), "strip buffers");
    SG_CUDA(h, cudaMemcpy(h->strip_cells, cells.data(), (size_t)n * sizeof(int4), cudaMemcpyHostToDevice), "strip cells");
    SG_CUDA(h, cudaMemcpy(h->strip_buf, params, (size_t)kParams * sizeof(float), cudaMemcpyHostToDevice), "strip parameters");
    h->strip_w = width;
    h->strip_n = n;
    return SGFD_OK;
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
    SG_CUDA(h, cudaMalloc(&dc, (size_t)n * sizeof(int4)), "feature scratch");
    cudaError_t e = cudaMalloc(&dX, (size_t)n * (kIn + 2) * sizeof(float));
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

int strip_cell_list(const Model &m, int w, std::vector<int4> &cells) {
    cells.clear();
    for (int z = 0; z < m.nzc; ++z)
        for (int y = 0; y < m.nyc; ++y)
            for (int x = 0; x < m.nxc; ++x) {
                const bool in = x < w || y < w || z < w || x >= m.nxc - w || y >= m.nyc - w || z >= m.nzc - w;
                if (in) cells.push_back(make_int4(x, y, z, 0));
            }
    return (int)cells.size();
}

cudaError_t strip_prepare() {
    return cudaFuncSetAttribute(k_strip_mlp, cudaFuncAttributeMaxDynamicSharedMemorySize, kParams * (int)sizeof(float));
}

cudaError_t launch_strip(const Model &m, int w, const int4 *cells, int n, const float *params, float *delta,
                         cudaStream_t s) {
    k_strip_mlp<<<cdiv(n, 128), 128, kParams * sizeof(float), s>>>(m, w, cells, n, params, delta);
    k_strip_apply<<<cdiv(n, 256), 256, 0, s>>>(m, cells, n, delta);
    return cudaGetLastError();
}

int mlp_params() { return kParams; }

}  // namespace sgfd
