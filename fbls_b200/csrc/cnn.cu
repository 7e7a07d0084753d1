// Kernels of the proposal network (the learned pruning of the search): a small 1D
// CNN over the coarse periodogram, trained and run on the GPU.
//
// Activations are laid out channel-major, [C][B][T] (channel, curve, position),
// so every convolution over a batch is one GEMM over an im2col copy of its
// input (Xcol [Ci*KW][B*T]):
//   forward        Y   = W   . Xcol     (Co x B*T, K = Ci * KW)
//   input grad     dXc = W^T . dY       (Ci*KW x B*T, K = Co), then col2im
//   weight grad    dW  = dY  . Xcol^T   (Co x Ci*KW, K = B * T)
// k_gemm_bf16 computes all three: operands are f32 in memory with arbitrary
// strides, staged into shared memory as bf16, multiplied on the tensor cores
// with mma.sync m16n8k16 (bf16 inputs, f32 accumulation) and written as f32.
// The network is a few MFLOP per curve, so these tiles are sized for
// simplicity, not for peak throughput.
#include <atomic>
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/fbls_b200.h"

namespace {

constexpr int BM = 64, BN = 64, BK = 32;
constexpr int GEMM_THREADS = 128;  // 4 warps, each a 32 x 32 block of C

struct GemmArgs {
    const float* A;
    const float* B;
    float* C;
    int M, N, K;
    long long sam, sak, sab;  // A(m, k) = A[m*sam + k*sak + b*sab]
    long long sbk, sbn, sbb;  // B(k, n)
    long long scm, scn, scb;  // C(m, n)
    float alpha, beta;        // C = alpha A B + beta C
};

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}

__global__ void __launch_bounds__(GEMM_THREADS) k_gemm_bf16(GemmArgs g) {
    // As[m][k] and Bs[n][k] (both k-contiguous: the mma fragments read pairs
    // along k), padded by 8 bf16 per row against bank conflicts.
    __shared__ __nv_bfloat16 As[BM][BK + 8];
    __shared__ __nv_bfloat16 Bs[BN][BK + 8];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN, b = blockIdx.z;
    const float* A = g.A + (long long)b * g.sab;
    const float* B = g.B + (long long)b * g.sbb;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    const int gid = lane >> 2, tig = lane & 3;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int r = 0; r < 4; r++) acc[i][j][r] = 0.f;

    for (int k0 = 0; k0 < g.K; k0 += BK) {
        for (int e = tid; e < BM * BK; e += GEMM_THREADS) {
            const int mm = e / BK, kk = e % BK;
            const int m = m0 + mm, k = k0 + kk;
            const float v = (m < g.M && k < g.K) ? A[(long long)m * g.sam + (long long)k * g.sak] : 0.f;
            As[mm][kk] = __float2bfloat16_rn(v);
        }
        for (int e = tid; e < BN * BK; e += GEMM_THREADS) {
            const int nn = e / BK, kk = e % BK;
            const int n = n0 + nn, k = k0 + kk;
            const float v = (n < g.N && k < g.K) ? B[(long long)k * g.sbk + (long long)n * g.sbn] : 0.f;
            Bs[nn][kk] = __float2bfloat16_rn(v);
        }
        __syncthreads();
#pragma unroll
        for (int ks = 0; ks < BK; ks += 16) {
            uint32_t af[2][4], bf[4][2];
#pragma unroll
            for (int i = 0; i < 2; i++) {
                const int r = wm + i * 16 + gid;
                af[i][0] = *reinterpret_cast<const uint32_t*>(&As[r][ks + tig * 2]);
                af[i][1] = *reinterpret_cast<const uint32_t*>(&As[r + 8][ks + tig * 2]);
                af[i][2] = *reinterpret_cast<const uint32_t*>(&As[r][ks + tig * 2 + 8]);
                af[i][3] = *reinterpret_cast<const uint32_t*>(&As[r + 8][ks + tig * 2 + 8]);
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int c = wn + j * 8 + gid;
                bf[j][0] = *reinterpret_cast<const uint32_t*>(&Bs[c][ks + tig * 2]);
                bf[j][1] = *reinterpret_cast<const uint32_t*>(&Bs[c][ks + tig * 2 + 8]);
            }
#pragma unroll
            for (int i = 0; i < 2; i++)
#pragma unroll
                for (int j = 0; j < 4; j++)
                    asm volatile(
                        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
                        "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};"
                        : "+f"(acc[i][j][0]), "+f"(acc[i][j][1]), "+f"(acc[i][j][2]), "+f"(acc[i][j][3])
                        : "r"(af[i][0]), "r"(af[i][1]), "r"(af[i][2]), "r"(af[i][3]), "r"(bf[j][0]),
                          "r"(bf[j][1]));
        }
        __syncthreads();
    }
    float* C = g.C + (long long)b * g.scb;
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int r = 0; r < 4; r++) {
                const int m = m0 + wm + i * 16 + gid + (r >= 2 ? 8 : 0);
                const int n = n0 + wn + j * 8 + tig * 2 + (r & 1);
                if (m < g.M && n < g.N) {
                    float* c = C + (long long)m * g.scm + (long long)n * g.scn;
                    const float prev = g.beta != 0.f ? g.beta * *c : 0.f;
                    *c = g.alpha * acc[i][j][r] + prev;
                }
            }
}

// Xcol[ci*KW + k][b][t] = X[ci][b][t + k - R], zero outside [0, T).
__global__ void k_im2col(const float* X, float* Xc, int B, int Ci, int T, int KW, int R) {
    const long long total = (long long)B * Ci * KW * T;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int t = (int)(e % T);
        const long long r = e / T;
        const int b = (int)(r % B);
        const long long ck = r / B;  // ci * KW + k
        const int k = (int)(ck % KW);
        const long long ci = ck / KW;
        const int s = t + k - R;
        Xc[e] = (s >= 0 && s < T) ? X[(ci * B + b) * T + s] : 0.f;
    }
}

// dX[ci][b][s] = sum_k dXcol[ci*KW + k][b][s - k + R].
__global__ void k_col2im(const float* dXc, float* dX, int B, int Ci, int T, int KW, int R) {
    const long long total = (long long)B * Ci * T;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int s = (int)(e % T);
        const long long r = e / T;
        const int b = (int)(r % B);
        const long long ci = r / B;
        float v = 0.f;
        for (int k = 0; k < KW; k++) {
            const int t = s - k + R;
            if (t >= 0 && t < T) v += dXc[(((ci * KW + k) * B) + b) * T + t];
        }
        dX[e] = v;
    }
}

// Z[c][b][u] = max over t in [u*P, u*P + P) of relu(Y[c][b][t] + bias[c]);
// idx keeps the window offset of the maximum (first one).
__global__ void k_bias_relu_pool(const float* Y, const float* bias, float* Z, uint8_t* idx, int B, int C, int T,
                                 int P) {
    const int U = T / P;
    const long long total = (long long)B * C * U;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int u = (int)(e % U);
        const long long bc = e / U;  // c * B + b
        const int c = (int)(bc / B);
        const float* y = Y + bc * T + (long long)u * P;
        float best = -1.f;
        int at = 0;
        for (int i = 0; i < P; i++) {
            const float v = fmaxf(y[i] + bias[c], 0.f);
            if (v > best) {
                best = v;
                at = i;
            }
        }
        Z[e] = best;
        idx[e] = (uint8_t)at;
    }
}

// dY[c][b][t] = dZ at the window's maximum when that maximum is positive
// (the ReLU passed it), else 0; dbias[c] += sum of dY (atomic).
__global__ void k_bias_relu_pool_bwd(const float* dZ, const float* Z, const uint8_t* idx, float* dY, float* dbias,
                                     int B, int C, int T, int P) {
    const int U = T / P;
    const long long total = (long long)B * C * U;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int u = (int)(e % U);
        const long long bc = e / U;  // c * B + b
        const int c = (int)(bc / B);
        float* y = dY + bc * T + (long long)u * P;
        const float g = Z[e] > 0.f ? dZ[e] : 0.f;
        for (int i = 0; i < P; i++) y[i] = (i == idx[e]) ? g : 0.f;
        if (g != 0.f) atomicAdd(&dbias[c], g);
    }
}

// GELU, x Phi(x) with the normal CDF Phi from CUDA's erff, and its
// derivative Phi(x) + x phi(x).
__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
    return 0.5f * (1.f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

// Z[c][b][u] = max over t in [u*P, u*P + P) of gelu(Y[c][b][t] + bias[c]);
// idx keeps the window offset of the maximum (first one). P = 1 is GELU alone.
__global__ void k_bias_gelu_pool(const float* Y, const float* bias, float* Z, uint8_t* idx, int B, int C, int T,
                                 int P) {
    const int U = T / P;
    const long long total = (long long)B * C * U;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int u = (int)(e % U);
        const long long bc = e / U;  // c * B + b
        const int c = (int)(bc / B);
        const float* y = Y + bc * T + (long long)u * P;
        float best = gelu(y[0] + bias[c]);
        int at = 0;
        for (int i = 1; i < P; i++) {
            const float v = gelu(y[i] + bias[c]);
            if (v > best) {
                best = v;
                at = i;
            }
        }
        Z[e] = best;
        idx[e] = (uint8_t)at;
    }
}

// dY[c][b][t] = dZ gelu'(Y + bias) at the window's maximum, else 0; dbias[c]
// += sum of dY (one atomic per thread and element with a nonzero gradient).
__global__ void k_bias_gelu_pool_bwd(const float* dZ, const float* Y, const uint8_t* idx, const float* bias, float* dY,
                                     float* dbias, int B, int C, int T, int P) {
    const int U = T / P;
    const long long total = (long long)B * C * U;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int u = (int)(e % U);
        const long long bc = e / U;  // c * B + b
        const int c = (int)(bc / B);
        const long long base = bc * T + (long long)u * P;
        const int at = idx[e];
        const float g = dZ[e] * gelu_grad(Y[base + at] + bias[c]);
        for (int i = 0; i < P; i++) dY[base + i] = (i == at) ? g : 0.f;
        if (g != 0.f) atomicAdd(&dbias[c], g);
    }
}

// Head: h[b][t] = sum_c wh[c] Z[c][b][t] + bh; logits[b][j] = mean of h over
// t in [j*G, j*G + G); softmax cross-entropy with label[b] (or no loss when
// labels is null): loss[b], dlogits[b][j] = (softmax - onehot) / B.
__global__ void k_head(const float* Z, const float* wh, const float* bh, const int* labels, float* logits,
                       float* loss, float* dlogits, int B, int C, int T, int G) {
    const int b = blockIdx.x;
    const int J = T / G;
    extern __shared__ float s_logit[];
    for (int j = threadIdx.x; j < J; j += blockDim.x) {
        float acc = 0.f;
        for (int t = j * G; t < j * G + G; t++) {
            float h = bh[0];
            for (int c = 0; c < C; c++) h += wh[c] * Z[((long long)c * B + b) * T + t];
            acc += h;
        }
        s_logit[j] = acc / (float)G;
        logits[(long long)b * J + j] = s_logit[j];
    }
    __syncthreads();
    if (labels == nullptr || threadIdx.x != 0) return;
    float mx = s_logit[0];
    for (int j = 1; j < J; j++) mx = fmaxf(mx, s_logit[j]);
    float sum = 0.f;
    for (int j = 0; j < J; j++) sum += expf(s_logit[j] - mx);
    const int y = labels[b];
    loss[b] = logf(sum) + mx - s_logit[y];
    for (int j = 0; j < J; j++)
        dlogits[(long long)b * J + j] = (expf(s_logit[j] - mx) / sum - (j == y ? 1.f : 0.f)) / (float)B;
}

// Head backward: dh[b][t] = dlogits[b][t/G] / G; dZ[c][b][t] = wh[c] dh[b][t];
// dwh[c] += sum_{b,t} dh Z; dbh += sum dh (atomics per block).
__global__ void k_head_bwd(const float* Z, const float* wh, const float* dlogits, float* dZ, float* dwh, float* dbh,
                           int B, int C, int T, int G) {
    const int b = blockIdx.x;
    const int J = T / G;
    for (int c = threadIdx.x; c < C; c += blockDim.x) {
        float acc = 0.f;
        for (int t = 0; t < T; t++) {
            const float dh = dlogits[(long long)b * J + t / G] / (float)G;
            acc += dh * Z[((long long)c * B + b) * T + t];
            dZ[((long long)c * B + b) * T + t] = wh[c] * dh;
        }
        atomicAdd(&dwh[c], acc);
    }
    if (threadIdx.x == 0) {
        float acc = 0.f;
        for (int j = 0; j < J; j++) acc += dlogits[(long long)b * J + j];
        atomicAdd(dbh, acc);
    }
}

// Adam (Kingma & Ba 2015) with bias correction: step t >= 1.
__global__ void k_adam(float* w, const float* g, float* m, float* v, long long n, float lr, float b1, float b2,
                       float eps, int t) {
    const float c1 = 1.f - powf(b1, (float)t), c2 = 1.f - powf(b2, (float)t);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        m[i] = b1 * m[i] + (1.f - b1) * g[i];
        v[i] = b2 * v[i] + (1.f - b2) * g[i] * g[i];
        w[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + eps);
    }
}

// AdamW (Loshchilov & Hutter 2019): Adam with bias correction and the weight
// decay decoupled from the gradient, w -= lr (m_hat / (sqrt(v_hat) + eps) +
// wd w); step t >= 1.
__global__ void k_adamw(float* w, const float* g, float* m, float* v, long long n, float lr, float b1, float b2,
                        float eps, float wd, int t) {
    const float c1 = 1.f - powf(b1, (float)t), c2 = 1.f - powf(b2, (float)t);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        m[i] = b1 * m[i] + (1.f - b1) * g[i];
        v[i] = b2 * v[i] + (1.f - b2) * g[i] * g[i];
        w[i] -= lr * ((m[i] / c1) / (sqrtf(v[i] / c2) + eps) + wd * w[i]);
    }
}

// Grid of a grid-stride elementwise kernel: one CTA of 256 threads per 256
// elements, at most 64 CTAs per SM of the current device (its SM count read
// once per device, so that launches being captured into a graph make no
// device queries).
int grid_for(long long total) {
    static std::atomic<int> sm_count[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) dev = -1;
    int sms = dev >= 0 ? sm_count[dev].load(std::memory_order_relaxed) : 0;
    if (sms < 1) {
        if (dev < 0 || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1)
            sms = 1;
        else
            sm_count[dev].store(sms, std::memory_order_relaxed);
    }
    const long long cap = 64LL * sms;
    long long b = (total + 255) / 256;
    return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

int status(cudaError_t e) { return e == cudaSuccess ? FBLS_OK : FBLS_ERR_CUDA; }

}  // namespace

extern "C" {

int fbls_nn_gemm(const float* A, const float* B, float* C, int M, int N, int K, long long sam, long long sak,
                 long long sab, long long sbk, long long sbn, long long sbb, long long scm, long long scn,
                 long long scb, int batch, float alpha, float beta, void* stream) {
    if (M < 1 || N < 1 || K < 1 || batch < 1 || !A || !B || !C) return FBLS_ERR_ARGUMENT;
    GemmArgs g{A, B, C, M, N, K, sam, sak, sab, sbk, sbn, sbb, scm, scn, scb, alpha, beta};
    dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM, batch);
    if (grid.y > 65535 || grid.z > 65535) return FBLS_ERR_ARGUMENT;
    k_gemm_bf16<<<grid, GEMM_THREADS, 0, static_cast<cudaStream_t>(stream)>>>(g);
    return status(cudaGetLastError());
}

int fbls_nn_im2col(const float* X, float* Xc, int B, int Ci, int T, int KW, int R, void* stream) {
    if (B < 1 || Ci < 1 || T < 1 || KW < 1 || R < 0 || R >= KW) return FBLS_ERR_ARGUMENT;
    k_im2col<<<grid_for((long long)B * Ci * KW * T), 256, 0, static_cast<cudaStream_t>(stream)>>>(X, Xc, B, Ci, T,
                                                                                               KW, R);
    return status(cudaGetLastError());
}

int fbls_nn_col2im(const float* dXc, float* dX, int B, int Ci, int T, int KW, int R, void* stream) {
    if (B < 1 || Ci < 1 || T < 1 || KW < 1 || R < 0 || R >= KW) return FBLS_ERR_ARGUMENT;
    k_col2im<<<grid_for((long long)B * Ci * T), 256, 0, static_cast<cudaStream_t>(stream)>>>(dXc, dX, B, Ci, T, KW,
                                                                                         R);
    return status(cudaGetLastError());
}

int fbls_nn_bias_relu_pool(const float* Y, const float* bias, float* Z, uint8_t* idx, int B, int C, int T, int P,
                           void* stream) {
    if (B < 1 || C < 1 || P < 1 || P > 255 || T % P) return FBLS_ERR_ARGUMENT;
    k_bias_relu_pool<<<grid_for((long long)B * C * (T / P)), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        Y, bias, Z, idx, B, C, T, P);
    return status(cudaGetLastError());
}

int fbls_nn_bias_relu_pool_bwd(const float* dZ, const float* Z, const uint8_t* idx, float* dY, float* dbias, int B,
                               int C, int T, int P, void* stream) {
    if (B < 1 || C < 1 || P < 1 || P > 255 || T % P) return FBLS_ERR_ARGUMENT;
    k_bias_relu_pool_bwd<<<grid_for((long long)B * C * (T / P)), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        dZ, Z, idx, dY, dbias, B, C, T, P);
    return status(cudaGetLastError());
}

int fbls_nn_bias_gelu_pool(const float* Y, const float* bias, float* Z, uint8_t* idx, int B, int C, int T, int P,
                           void* stream) {
    if (B < 1 || C < 1 || P < 1 || P > 255 || T % P) return FBLS_ERR_ARGUMENT;
    k_bias_gelu_pool<<<grid_for((long long)B * C * (T / P)), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        Y, bias, Z, idx, B, C, T, P);
    return status(cudaGetLastError());
}

int fbls_nn_bias_gelu_pool_bwd(const float* dZ, const float* Y, const uint8_t* idx, const float* bias, float* dY,
                               float* dbias, int B, int C, int T, int P, void* stream) {
    if (B < 1 || C < 1 || P < 1 || P > 255 || T % P) return FBLS_ERR_ARGUMENT;
    k_bias_gelu_pool_bwd<<<grid_for((long long)B * C * (T / P)), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        dZ, Y, idx, bias, dY, dbias, B, C, T, P);
    return status(cudaGetLastError());
}

int fbls_nn_adamw(float* w, const float* g, float* m, float* v, long long n, float lr, float b1, float b2, float eps,
                  float wd, int t, void* stream) {
    if (n < 1 || t < 1) return FBLS_ERR_ARGUMENT;
    k_adamw<<<grid_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(w, g, m, v, n, lr, b1, b2, eps, wd, t);
    return status(cudaGetLastError());
}

int fbls_nn_head(const float* Z, const float* wh, const float* bh, const int* labels, float* logits, float* loss,
                 float* dlogits, int B, int C, int T, int G, void* stream) {
    if (B < 1 || C < 1 || G < 1 || T % G || T / G > 4096) return FBLS_ERR_ARGUMENT;
    k_head<<<B, 128, (T / G) * sizeof(float), static_cast<cudaStream_t>(stream)>>>(Z, wh, bh, labels, logits, loss,
                                                                                 dlogits, B, C, T, G);
    return status(cudaGetLastError());
}

int fbls_nn_head_bwd(const float* Z, const float* wh, const float* dlogits, float* dZ, float* dwh, float* dbh, int B,
                     int C, int T, int G, void* stream) {
    if (B < 1 || C < 1 || G < 1 || T % G) return FBLS_ERR_ARGUMENT;
    k_head_bwd<<<B, 64, 0, static_cast<cudaStream_t>(stream)>>>(Z, wh, dlogits, dZ, dwh, dbh, B, C, T, G);
    return status(cudaGetLastError());
}

int fbls_nn_adam(float* w, const float* g, float* m, float* v, long long n, float lr, float b1, float b2, float eps,
                 int t, void* stream) {
    if (n < 1 || t < 1) return FBLS_ERR_ARGUMENT;
    k_adam<<<grid_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(w, g, m, v, n, lr, b1, b2, eps, t);
    return status(cudaGetLastError());
}

}  // extern "C"
