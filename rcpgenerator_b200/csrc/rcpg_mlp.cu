// Learned warm start: a small MLP (BF16 weights and activations, FP32
// accumulation, FP32 master weights) mapping size-distribution descriptors to
// a predicted phi_J and a growth schedule. Hand-written training and inference
// kernels: a strided tensor-core GEMM (mma.sync BF16 -> FP32), GELU, mean
// squared error, Adam.
//
// Parameters of an L-layer MLP with widths w[0..L] are packed in one FP32
// array: layer l holds W_l [w[l+1] x w[l]] row-major, then b_l [w[l+1]]. The
// hidden layers use GELU (0.5 x (1 + erf(x / sqrt 2))), the output is linear.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/rcpg.h"

namespace {

// Tensor-core GEMM: C[m, n] = sum_k A[m*sam + k*sak] * B[k*sbk + n*sbn] (+ bias[n]).
// A 64x64 tile of C per block of 4 warps (2x2), each warp 32x32 as 2x4
// mma.sync.m16n8k16 BF16 tiles with FP32 accumulators. Any operand strides:
// every K step of 16 stages the A (m, k) and B (n, k) slices in shared memory,
// zero-filled outside the matrices, with rows padded to 24 elements (12
// words) so that the fragment loads of a warp fall in distinct banks.
constexpr int kBM = 64, kBN = 64, kBK = 16, kPad = 24, kGemmThreads = 128;

__device__ __forceinline__ std::uint32_t lds_pair(const __nv_bfloat16* p) {
    return *reinterpret_cast<const std::uint32_t*>(p);
}

__global__ void __launch_bounds__(kGemmThreads)
    k_gemm_bf16(int M, int N, int K, const __nv_bfloat16* __restrict__ A, long long sam, long long sak,
                const __nv_bfloat16* __restrict__ B, long long sbk, long long sbn, float* __restrict__ C,
                long long ldc, const float* __restrict__ bias) {
    __shared__ __align__(16) __nv_bfloat16 As[kBM][kPad];
    __shared__ __align__(16) __nv_bfloat16 Bs[kBN][kPad];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.0f;
    const __nv_bfloat16 zero = __float2bfloat16(0.0f);
    for (int k0 = 0; k0 < K; k0 += kBK) {
        // stage: 64x16 elements of each operand, 8 per thread
#pragma unroll
        for (int r = 0; r < (kBM * kBK) / kGemmThreads; ++r) {
            const int e = tid + r * kGemmThreads;
            const int row = e / kBK, kk = e % kBK;
            const int m = m0 + row, n = n0 + row, k = k0 + kk;
            As[row][kk] = (m < M && k < K) ? A[m * sam + k * sak] : zero;
            Bs[row][kk] = (n < N && k < K) ? B[k * sbk + n * sbn] : zero;
        }
        __syncthreads();
        std::uint32_t af[2][4], bf[4][2];
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int r0 = wm + i * 16 + g;
            af[i][0] = lds_pair(&As[r0][2 * t]);
            af[i][1] = lds_pair(&As[r0 + 8][2 * t]);
            af[i][2] = lds_pair(&As[r0][2 * t + 8]);
            af[i][3] = lds_pair(&As[r0 + 8][2 * t + 8]);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int c0 = wn + j * 8 + g;
            bf[j][0] = lds_pair(&Bs[c0][2 * t]);
            bf[j][1] = lds_pair(&Bs[c0][2 * t + 8]);
        }
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
                asm volatile(
                    "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
                    "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};\n"
                    : "+f"(acc[i][j][0]), "+f"(acc[i][j][1]), "+f"(acc[i][j][2]), "+f"(acc[i][j][3])
                    : "r"(af[i][0]), "r"(af[i][1]), "r"(af[i][2]), "r"(af[i][3]), "r"(bf[j][0]), "r"(bf[j][1]));
        __syncthreads();
    }
    // epilogue: c0, c1 at (g, 2t..2t+1), c2, c3 at (g+8, 2t..2t+1) of each 16x8 tile
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int m = m0 + wm + i * 16 + g + (r >= 2 ? 8 : 0);
                const int n = n0 + wn + j * 8 + 2 * t + (r & 1);
                if (m < M && n < N) C[m * ldc + n] = acc[i][j][r] + (bias ? bias[n] : 0.0f);
            }
}

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
    return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

// activation of a layer's pre-activations z: a = gelu(z) (hidden) or z (output), stored BF16
__global__ void k_act(int n, const float* __restrict__ z, __nv_bfloat16* __restrict__ a, int hidden) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = __float2bfloat16(hidden ? gelu(z[i]) : z[i]);
}

// output layer: loss terms and dL/dz = 2 (y - t) / (B * O), BF16
__global__ void k_mse(int B, int O, const float* __restrict__ z, const float* __restrict__ t,
                      const float* __restrict__ wt, __nv_bfloat16* __restrict__ dz, float* __restrict__ lterm) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B * O) return;
    const float w = wt ? wt[i % O] : 1.0f;
    const float d = z[i] - t[i];
    lterm[i] = w * d * d;
    dz[i] = __float2bfloat16(2.0f * w * d / static_cast<float>(B * O));
}

// dz = da * gelu'(z), BF16
__global__ void k_gelu_bwd(int n, const float* __restrict__ da, const float* __restrict__ z,
                           __nv_bfloat16* __restrict__ dz) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dz[i] = __float2bfloat16(da[i] * gelu_grad(z[i]));
}

// db[o] = sum_b dz[b, o] (FP32, b ascending)
__global__ void k_bias_grad(int B, int O, const __nv_bfloat16* __restrict__ dz, float* __restrict__ db) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= O) return;
    float s = 0.0f;
    for (int b = 0; b < B; ++b) s += __bfloat162float(dz[b * O + o]);
    db[o] = s;
}

__global__ void k_to_bf16(int n, const float* __restrict__ x, __nv_bfloat16* __restrict__ y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = __float2bfloat16(x[i]);
}

// Adam on the FP32 master weights, then the BF16 copy
__global__ void k_adam(int n, float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ g, float lr, float b1, float b2, float c1, float c2,
                       __nv_bfloat16* __restrict__ wb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + 1e-8f);
    w[i] = wi;
    wb[i] = __float2bfloat16(wi);
}

void gemm(cudaStream_t st, int M, int N, int K, const __nv_bfloat16* A, long long sam, long long sak,
          const __nv_bfloat16* B, long long sbk, long long sbn, float* C, long long ldc, const float* bias) {
    dim3 grid((N + kBN - 1) / kBN, (M + kBM - 1) / kBM);
    k_gemm_bf16<<<grid, kGemmThreads, 0, st>>>(M, N, K, A, sam, sak, B, sbk, sbn, C, ldc, bias);
}

unsigned blocks(long long n) { return static_cast<unsigned>((n + 255) / 256); }

std::size_t param_count(const int32_t* w, int L) {
    std::size_t n = 0;
    for (int l = 0; l < L; ++l) n += static_cast<std::size_t>(w[l + 1]) * w[l] + w[l + 1];
    return n;
}

// Scratch of one forward/backward pass, carved from the caller's workspace.
struct Work {
    std::vector<__nv_bfloat16*> act;  // act[0] = input, act[l+1] = output of layer l (BF16)
    std::vector<float*> z;            // pre-activations of layer l (FP32)
    float* da;                        // FP32 gradient w.r.t. an activation
    __nv_bfloat16* dz;                // BF16 gradient w.r.t. a pre-activation
    __nv_bfloat16* dzp;               // the previous layer's
    float* lterm;
};

bool carve(void* ws, std::size_t ws_bytes, const int32_t* w, int L, int B, Work& wk) {
    auto* p = static_cast<unsigned char*>(ws);
    std::size_t used = 0;
    auto take = [&](std::size_t bytes) -> void* {
        used = (used + 255) & ~std::size_t{255};
        void* r = p + used;
        used += bytes;
        return r;
    };
    int wmax = 0;
    for (int l = 0; l <= L; ++l) wmax = w[l] > wmax ? w[l] : wmax;
    wk.act.resize(L + 1);
    wk.z.resize(L);
    for (int l = 0; l <= L; ++l) wk.act[l] = static_cast<__nv_bfloat16*>(take(static_cast<std::size_t>(B) * w[l] * 2));
    for (int l = 0; l < L; ++l) wk.z[l] = static_cast<float*>(take(static_cast<std::size_t>(B) * w[l + 1] * 4));
    wk.da = static_cast<float*>(take(static_cast<std::size_t>(B) * wmax * 4));
    wk.dz = static_cast<__nv_bfloat16*>(take(static_cast<std::size_t>(B) * wmax * 2));
    wk.dzp = static_cast<__nv_bfloat16*>(take(static_cast<std::size_t>(B) * wmax * 2));
    wk.lterm = static_cast<float*>(take(static_cast<std::size_t>(B) * w[L] * 4));
    return used <= ws_bytes;
}

void forward(cudaStream_t st, const int32_t* w, int L, int B, const __nv_bfloat16* wb, const float* w32,
             const float* X, Work& wk) {
    k_to_bf16<<<blocks(static_cast<long long>(B) * w[0]), 256, 0, st>>>(B * w[0], X, wk.act[0]);
    std::size_t off = 0;
    for (int l = 0; l < L; ++l) {
        const int I = w[l], O = w[l + 1];
        // z[b, o] = sum_i act[b, i] W[o, i] + bias[o]
        gemm(st, B, O, I, wk.act[l], I, 1, wb + off, 1, I, wk.z[l], O, w32 + off + static_cast<std::size_t>(O) * I);
        k_act<<<blocks(static_cast<long long>(B) * O), 256, 0, st>>>(B * O, wk.z[l], wk.act[l + 1], l + 1 < L);
        off += static_cast<std::size_t>(O) * I + O;
    }
}

int32_t fail(char* err, std::size_t errlen, int32_t code, const char* msg) {
    if (err && errlen) std::snprintf(err, errlen, "%s", msg);
    return code;
}

bool widths_ok(const int32_t* w, int L) {
    if (!w || L <= 0) return false;
    for (int l = 0; l <= L; ++l)
        if (w[l] <= 0 || w[l] > (1 << 20)) return false;
    return true;
}

}  // namespace

extern "C" {

uint64_t rcpg_mlp_param_count(const int32_t* widths, int32_t layers) {
    return widths_ok(widths, layers) ? param_count(widths, layers) : 0;
}

uint64_t rcpg_mlp_workspace_bytes(const int32_t* widths, int32_t layers, int32_t batch) {
    if (!widths_ok(widths, layers) || batch <= 0) return 0;
    int wmax = 0;
    std::size_t b = 0;
    for (int l = 0; l <= layers; ++l) {
        wmax = widths[l] > wmax ? widths[l] : wmax;
        b += static_cast<std::size_t>(batch) * widths[l] * 2 + 256;
    }
    for (int l = 0; l < layers; ++l) b += static_cast<std::size_t>(batch) * widths[l + 1] * 4 + 256;
    b += static_cast<std::size_t>(batch) * wmax * 8 + 3 * 256 + static_cast<std::size_t>(batch) * widths[layers] * 4 + 256;
    return b;
}

int32_t rcpg_mlp_forward(const int32_t* widths, int32_t layers, int32_t batch, const void* w_bf16,
                         const float* w_fp32, const float* X, float* Y, void* workspace,
                         uint64_t workspace_bytes, void* stream, char* err, size_t errlen) {
    if (!widths_ok(widths, layers) || batch <= 0 || !w_bf16 || !w_fp32 || !X || !Y || !workspace)
        return fail(err, errlen, RCPG_EINVAL, "rcpgenerator_b200: bad arguments to rcpg_mlp_forward");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Work wk;
    if (!carve(workspace, workspace_bytes, widths, layers, batch, wk))
        return fail(err, errlen, RCPG_EINVAL, "rcpgenerator_b200: MLP workspace too small");
    forward(st, widths, layers, batch, static_cast<const __nv_bfloat16*>(w_bf16), w_fp32, X, wk);
    cudaMemcpyAsync(Y, wk.z[layers - 1], static_cast<std::size_t>(batch) * widths[layers] * 4,
                    cudaMemcpyDeviceToDevice, st);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(err, errlen, RCPG_ECUDA, cudaGetErrorString(e));
    return RCPG_OK;
}

int32_t rcpg_mlp_train_step(const int32_t* widths, int32_t layers, int32_t batch, float* w_fp32,
                            void* w_bf16, float* adam_m, float* adam_v, float* grad, const float* X,
                            const float* T, const float* out_weight, float lr, int32_t step,
                            float* loss_terms, void* workspace, uint64_t workspace_bytes, void* stream,
                            char* err, size_t errlen) {
    if (!widths_ok(widths, layers) || batch <= 0 || !w_fp32 || !w_bf16 || !grad || !X || !T || !workspace)
        return fail(err, errlen, RCPG_EINVAL, "rcpgenerator_b200: bad arguments to rcpg_mlp_train_step");
    if (adam_m && adam_v && lr > 0.0f && step < 1)
        return fail(err, errlen, RCPG_EINVAL, "rcpgenerator_b200: the Adam step counter starts at 1");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Work wk;
    if (!carve(workspace, workspace_bytes, widths, layers, batch, wk))
        return fail(err, errlen, RCPG_EINVAL, "rcpgenerator_b200: MLP workspace too small");
    auto* wb = static_cast<__nv_bfloat16*>(w_bf16);
    forward(st, widths, layers, batch, wb, w_fp32, X, wk);
    const int O = widths[layers];
    k_mse<<<blocks(static_cast<long long>(batch) * O), 256, 0, st>>>(batch, O, wk.z[layers - 1], T, out_weight,
                                                                      wk.dz, wk.lterm);
    // offsets of the layers in the packed parameters
    std::vector<std::size_t> off(layers + 1, 0);
    for (int l = 0; l < layers; ++l) off[l + 1] = off[l] + static_cast<std::size_t>(widths[l + 1]) * widths[l] + widths[l + 1];
    for (int l = layers - 1; l >= 0; --l) {
        const int I = widths[l], Ol = widths[l + 1];
        float* gW = grad + off[l];
        float* gb = gW + static_cast<std::size_t>(Ol) * I;
        // dW[o, i] = sum_b dz[b, o] act[b, i]
        gemm(st, Ol, I, batch, wk.dz, 1, Ol, wk.act[l], I, 1, gW, I, nullptr);
        k_bias_grad<<<blocks(Ol), 256, 0, st>>>(batch, Ol, wk.dz, gb);
        if (l > 0) {
            // da[b, i] = sum_o dz[b, o] W[o, i]; dz_prev = da * gelu'(z_prev)
            gemm(st, batch, I, Ol, wk.dz, Ol, 1, wb + off[l], I, 1, wk.da, I, nullptr);
            k_gelu_bwd<<<blocks(static_cast<long long>(batch) * I), 256, 0, st>>>(batch * I, wk.da, wk.z[l - 1], wk.dzp);
            std::swap(wk.dz, wk.dzp);
        }
    }
    if (loss_terms)
        cudaMemcpyAsync(loss_terms, wk.lterm, static_cast<std::size_t>(batch) * O * 4, cudaMemcpyDeviceToDevice, st);
    if (adam_m && adam_v && lr > 0.0f) {
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.0f - std::pow(b1, static_cast<float>(step)), c2 = 1.0f - std::pow(b2, static_cast<float>(step));
        const int n = static_cast<int>(off[layers]);
        k_adam<<<blocks(n), 256, 0, st>>>(n, w_fp32, adam_m, adam_v, grad, lr, b1, b2, c1, c2, wb);
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(err, errlen, RCPG_ECUDA, cudaGetErrorString(e));
    return RCPG_OK;
}

int32_t rcpg_mlp_to_bf16(uint64_t n, const float* x, void* y, void* stream) {
    if (!x || !y) return RCPG_EINVAL;
    k_to_bf16<<<blocks(static_cast<long long>(n)), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<int>(n), x, static_cast<__nv_bfloat16*>(y));
    return cudaGetLastError() == cudaSuccess ? RCPG_OK : RCPG_ECUDA;
}

}  // extern "C"
