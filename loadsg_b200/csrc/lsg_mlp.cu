// Learned diagonal preconditioner: a small MLP (F inputs, three hidden layers
// of 64 with ReLU, one output) with BF16 weights and FP32 accumulation,
// trained on the GPU by the kernels below (forward, backward, Adam).
//
// Work is organised in tiles of 64 rows: a CTA keeps the tile's inputs and all
// hidden activations in shared memory.  The three hidden layers run on the
// tensor cores: mma.sync m16n8k16 with BF16 A (the layer input, rounded to
// BF16) and BF16 B (the weights), FP32 accumulation, bias and ReLU in FP32; each
// of the CTA's 8 warps owns a 16 x 32 block of the 64 x 64 layer output.  The
// output layer (64 -> 1) and the backward pass run on the CUDA cores with the
// same rounded activations; the backward pass forms the weight gradients of
// the tile as activation^T x delta products, adding them to the global
// gradient with one atomic per parameter per tile.
//
// Parameter layout (FP32 master copy, flat):
//   W1[64][F] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[64] b4[1]
// The forward and backward passes use the BF16-rounded weights (round to
// nearest even), the Adam update works on the FP32 master copy.
#include "../../include/lsg.h"

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

namespace {

constexpr int H = 64;      // hidden width
constexpr int TR = 64;     // rows per tile
constexpr int MAXF = 64;   // max input features

thread_local std::string g_mlp_err;
int mfail(int code, const std::string& m) {
    g_mlp_err = m;
    return code;
}

struct Layout {
    int F;
    int64_t w1, b1, w2, b2, w3, b3, w4, b4, total;
    __host__ __device__ explicit Layout(int f) : F(f) {
        w1 = 0;
        b1 = w1 + (int64_t)H * F;
        w2 = b1 + H;
        b2 = w2 + H * H;
        w3 = b2 + H;
        b3 = w3 + H * H;
        w4 = b3 + H;
        b4 = w4 + H;
        total = b4 + 1;
    }
};

__device__ __forceinline__ float softplus(float o) { return o > 20.f ? o : log1pf(expf(o)); }
__device__ __forceinline__ float sigmoidf_(float o) { return 1.f / (1.f + expf(-o)); }

constexpr int LDH = H + 8;  // BF16 row stride of 64-wide operands (conflict-free fragment loads)
__host__ __device__ inline int ldx(int F) { return ((F + 15) / 16) * 16 + 8; }  // layer-1 input stride

// shared-memory tile of the network's weights (BF16 values widened to FP32)
// and, for the tensor cores, BF16 copies of the weights and layer inputs
struct Smem {
    float* W1;  // H*F
    float* W2;  // H*H
    float* W3;  // H*H
    float* W4;  // H
    float* b;   // 3H + 1
    float* X;   // TR*F
    float* A1;  // TR*H
    float* A2;
    float* A3;
    float* o;   // TR
    __nv_bfloat16* W1b;  // H x ldx(F), zero padded
    __nv_bfloat16* W2b;  // H x LDH
    __nv_bfloat16* W3b;
    __nv_bfloat16* Xb;   // TR x ldx(F), zero padded
    __nv_bfloat16* A1b;  // TR x LDH
    __nv_bfloat16* A2b;
};

__device__ Smem carve(float* base, int F) {
    Smem s;
    s.W1 = base;
    s.W2 = s.W1 + H * F;
    s.W3 = s.W2 + H * H;
    s.W4 = s.W3 + H * H;
    s.b = s.W4 + H;
    s.X = s.b + 3 * H + 1;
    s.A1 = s.X + TR * F;
    s.A2 = s.A1 + TR * H;
    s.A3 = s.A2 + TR * H;
    s.o = s.A3 + TR * H;
    s.W1b = reinterpret_cast<__nv_bfloat16*>(s.o + TR);
    s.W2b = s.W1b + H * ldx(F);
    s.W3b = s.W2b + H * LDH;
    s.Xb = s.W3b + H * LDH;
    s.A1b = s.Xb + TR * ldx(F);
    s.A2b = s.A1b + TR * LDH;
    return s;
}

size_t smem_bytes(int F) {
    return sizeof(float) * ((size_t)H * F + 2 * H * H + H + 3 * H + 1 + TR * F + 3 * TR * H + TR) +
           sizeof(__nv_bfloat16) * ((size_t)(H + TR) * ldx(F) + (size_t)(2 * H + 2 * TR) * LDH);
}

__device__ void load_weights(const __nv_bfloat16* wb, const float* p, Smem& s, int F) {
    Layout L(F);
    const int lx = ldx(F);
    for (int i = threadIdx.x; i < H * F; i += blockDim.x) s.W1[i] = __bfloat162float(wb[L.w1 + i]);
    for (int i = threadIdx.x; i < H * lx; i += blockDim.x) {
        int o = i / lx, k = i % lx;
        s.W1b[i] = k < F ? wb[L.w1 + o * F + k] : __float2bfloat16_rn(0.f);
    }
    for (int i = threadIdx.x; i < H * H; i += blockDim.x) {
        s.W2[i] = __bfloat162float(wb[L.w2 + i]);
        s.W3[i] = __bfloat162float(wb[L.w3 + i]);
        s.W2b[(i / H) * LDH + i % H] = wb[L.w2 + i];
        s.W3b[(i / H) * LDH + i % H] = wb[L.w3 + i];
    }
    for (int i = threadIdx.x; i < TR * lx; i += blockDim.x) s.Xb[i] = __float2bfloat16_rn(0.f);  // K padding
    for (int i = threadIdx.x; i < H; i += blockDim.x) {
        s.W4[i] = __bfloat162float(wb[L.w4 + i]);
        s.b[i] = p[L.b1 + i];
        s.b[H + i] = p[L.b2 + i];
        s.b[2 * H + i] = p[L.b3 + i];
    }
    if (threadIdx.x == 0) s.b[3 * H] = p[L.b4];
}

// D += A * B for one m16n8k16 tile: A 16 x 16 BF16 (row), B 16 x 8 BF16 (col), D FP32
__device__ __forceinline__ void mma_bf16(float* d, const uint32_t* a, const uint32_t* b) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// One hidden layer on the tensor cores: A[r][o] = relu(b[o] + sum_k W[o][k] In[r][k])
// for r < TR, o < H, K a multiple of 16 (In, W BF16 with row strides ldi, ldw).
// Warp w computes rows 16 (w & 3) .. +15 and columns 32 (w >> 2) .. +31.
// Af receives the result (rounded to BF16 when Ab is given, the next layer's
// input, so that Af holds exactly what that layer reads); Ab its BF16 copy.
__device__ void layer_tc(const __nv_bfloat16* In, int ldi, int K, const __nv_bfloat16* W, int ldw, const float* bias,
                         float* Af, __nv_bfloat16* Ab) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int r0 = (warp & 3) * 16, c0 = (warp >> 2) * 32;
    float acc[4][4];
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[j][q] = 0.f;
    for (int k0 = 0; k0 < K; k0 += 16) {
        uint32_t a[4];
        a[0] = *reinterpret_cast<const uint32_t*>(In + (r0 + g) * ldi + k0 + 2 * t);
        a[1] = *reinterpret_cast<const uint32_t*>(In + (r0 + g + 8) * ldi + k0 + 2 * t);
        a[2] = *reinterpret_cast<const uint32_t*>(In + (r0 + g) * ldi + k0 + 2 * t + 8);
        a[3] = *reinterpret_cast<const uint32_t*>(In + (r0 + g + 8) * ldi + k0 + 2 * t + 8);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int n = c0 + 8 * j + g;
            uint32_t b[2];
            b[0] = *reinterpret_cast<const uint32_t*>(W + n * ldw + k0 + 2 * t);
            b[1] = *reinterpret_cast<const uint32_t*>(W + n * ldw + k0 + 2 * t + 8);
            mma_bf16(acc[j], a, b);
        }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int col = c0 + 8 * j + 2 * t;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int r = r0 + g + (q >= 2 ? 8 : 0), c = col + (q & 1);
            float v = acc[j][q] + bias[c];
            v = v > 0.f ? v : 0.f;
            if (Ab) {
                __nv_bfloat16 vb = __float2bfloat16_rn(v);
                Ab[r * LDH + c] = vb;
                v = __bfloat162float(vb);
            }
            Af[r * H + c] = v;
        }
    }
}

__device__ void forward_tile(const float* __restrict__ X, int64_t row0, int64_t rows, Smem& s, int F) {
    const int lx = ldx(F);
    for (int e = threadIdx.x; e < TR * F; e += blockDim.x) {
        int64_t r = row0 + e / F;
        __nv_bfloat16 vb = __float2bfloat16_rn(r < rows ? X[r * F + e % F] : 0.f);
        s.Xb[(e / F) * lx + e % F] = vb;
        s.X[e] = __bfloat162float(vb);  // the layer-1 input as the tensor cores see it
    }
    __syncthreads();
    layer_tc(s.Xb, lx, ((F + 15) / 16) * 16, s.W1b, lx, s.b, s.A1, s.A1b);
    __syncthreads();
    layer_tc(s.A1b, LDH, H, s.W2b, LDH, s.b + H, s.A2, s.A2b);
    __syncthreads();
    layer_tc(s.A2b, LDH, H, s.W3b, LDH, s.b + 2 * H, s.A3, nullptr);
    __syncthreads();
    for (int r = threadIdx.x; r < TR; r += blockDim.x) {
        float acc = s.b[3 * H];
        for (int i = 0; i < H; ++i) acc = fmaf(s.W4[i], s.A3[r * H + i], acc);
        s.o[r] = acc;
    }
    __syncthreads();
}

__global__ void k_forward(const __nv_bfloat16* __restrict__ wb, const float* __restrict__ p, const float* __restrict__ X,
                          int64_t rows, int F, float* __restrict__ out) {
    extern __shared__ float sm[];
    Smem s = carve(sm, F);
    load_weights(wb, p, s, F);
    __syncthreads();
    for (int64_t row0 = (int64_t)blockIdx.x * TR; row0 < rows; row0 += (int64_t)gridDim.x * TR) {
        forward_tile(X, row0, rows, s, F);
        for (int r = threadIdx.x; r < TR; r += blockDim.x)
            if (row0 + r < rows) out[row0 + r] = s.o[r];
        __syncthreads();
    }
}

// Loss per row: (log softplus(o) - y)^2, mean over rows.  Adds d(mean loss)/dp
// to grad and the summed loss to *loss.
__global__ void k_backward(const __nv_bfloat16* __restrict__ wb, const float* __restrict__ p, const float* __restrict__ X,
                           const float* __restrict__ Y, int64_t rows, int F, float* __restrict__ grad,
                           float* __restrict__ loss) {
    extern __shared__ float sm[];
    Smem s = carve(sm, F);
    Layout L(F);
    load_weights(wb, p, s, F);
    __syncthreads();
    const float inv = 1.f / (float)rows;
    for (int64_t row0 = (int64_t)blockIdx.x * TR; row0 < rows; row0 += (int64_t)gridDim.x * TR) {
        forward_tile(X, row0, rows, s, F);
        // output delta: d/do (log sp(o) - y)^2 / rows
        for (int r = threadIdx.x; r < TR; r += blockDim.x) {
            float dout = 0.f;
            if (row0 + r < rows) {
                float o = s.o[r], sp = softplus(o), e = logf(sp) - Y[row0 + r];
                atomicAdd(loss, e * e);
                dout = 2.f * e * sigmoidf_(o) / sp * inv;
            }
            s.o[r] = dout;
        }
        __syncthreads();
        // layer 4: grads, and delta3 = W4 * dout masked by relu'(a3), stored over A3's
        for (int i = threadIdx.x; i < H; i += blockDim.x) {
            float g = 0.f;
            for (int r = 0; r < TR; ++r) g = fmaf(s.o[r], s.A3[r * H + i], g);
            atomicAdd(&grad[L.w4 + i], g);
        }
        if (threadIdx.x == 0) {
            float g = 0.f;
            for (int r = 0; r < TR; ++r) g += s.o[r];
            atomicAdd(&grad[L.b4], g);
        }
        __syncthreads();
        for (int e = threadIdx.x; e < TR * H; e += blockDim.x) {
            int r = e / H, i = e % H;
            s.A3[e] = s.A3[e] > 0.f ? s.W4[i] * s.o[r] : 0.f;  // delta3
        }
        __syncthreads();
        // layer 3: dW3[o][i] = sum_r delta3[r][o] a2[r][i]; db3 = sum_r delta3
        for (int e = threadIdx.x; e < H * H; e += blockDim.x) {
            int o = e / H, i = e % H;
            float g = 0.f;
            for (int r = 0; r < TR; ++r) g = fmaf(s.A3[r * H + o], s.A2[r * H + i], g);
            atomicAdd(&grad[L.w3 + e], g);
        }
        for (int o = threadIdx.x; o < H; o += blockDim.x) {
            float g = 0.f;
            for (int r = 0; r < TR; ++r) g += s.A3[r * H + o];
            atomicAdd(&grad[L.b3 + o], g);
        }
        __syncthreads();
        // delta2[r][i] = relu'(a2) * sum_o W3[o][i] delta3[r][o]  (written over A2 after use)
        {
            // compute into A1-sized scratch? A1 is still needed for dW2, so use X-free order:
            // first compute delta2 into registers per element and store into A2 after a barrier
            float tmp[TR * H / 256 + 1];
            int c = 0;
            for (int e = threadIdx.x; e < TR * H; e += blockDim.x, ++c) {
                int r = e / H, i = e % H;
                float acc = 0.f;
                for (int o = 0; o < H; ++o) acc = fmaf(s.W3[o * H + i], s.A3[r * H + o], acc);
                tmp[c] = s.A2[e] > 0.f ? acc : 0.f;
            }
            __syncthreads();
            c = 0;
            for (int e = threadIdx.x; e < TR * H; e += blockDim.x, ++c) s.A2[e] = tmp[c];
        }
        __syncthreads();
        // layer 2
        for (int e = threadIdx.x; e < H * H; e += blockDim.x) {
            int o = e / H, i = e % H;
            float g = 0.f;
            for (int r = 0; r < TR; ++r) g = fmaf(s.A2[r * H + o], s.A1[r * H + i], g);
            atomicAdd(&grad[L.w2 + e], g);
        }
        for (int o = threadIdx.x; o < H; o += blockDim.x) {
            float g = 0.f;
            for (int r = 0; r < TR; ++r) g += s.A2[r * H + o];
            atomicAdd(&grad[L.b2 + o], g);
        }
        __syncthreads();
        {
            float tmp[TR * H / 256 + 1];
            int c = 0;
            for (int e = threadIdx.x; e < TR * H; e += blockDim.x, ++c) {
                int r = e / H, i = e % H;
                float acc = 0.f;
                for (int o = 0; o < H; ++o) acc = fmaf(s.W2[o * H + i], s.A2[r * H + o], acc);
                tmp[c] = s.A1[e] > 0.f ? acc : 0.f;
            }
            __syncthreads();
            c = 0;
            for (int e = threadIdx.x; e < TR * H; e += blockDim.x, ++c) s.A1[e] = tmp[c];
        }
        __syncthreads();
        // layer 1
        for (int e = threadIdx.x; e < H * F; e += blockDim.x) {
            int o = e / F, i = e % F;
            float g = 0.f;
            for (int r = 0; r < TR; ++r) g = fmaf(s.A1[r * H + o], s.X[r * F + i], g);
            atomicAdd(&grad[L.w1 + e], g);
        }
        for (int o = threadIdx.x; o < H; o += blockDim.x) {
            float g = 0.f;
            for (int r = 0; r < TR; ++r) g += s.A1[r * H + o];
            atomicAdd(&grad[L.b1 + o], g);
        }
        __syncthreads();
    }
}

__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       int64_t n, float lr, float b1, float b2, float eps, float c1, float c2,
                       __nv_bfloat16* __restrict__ wb) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    float gi = g[i];
    float mi = b1 * m[i] + (1.f - b1) * gi;
    float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    p[i] = pi;
    wb[i] = __float2bfloat16_rn(pi);
}

__global__ void k_to_bf16(const float* __restrict__ p, int64_t n, __nv_bfloat16* __restrict__ wb) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) wb[i] = __float2bfloat16_rn(p[i]);
}

}  // namespace

struct lsg_mlp {
    int F = 0;
    int64_t np = 0;
    float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr, *loss = nullptr;
    __nv_bfloat16* wb = nullptr;
    int64_t step = 0;
    ~lsg_mlp() {
        cudaFree(p);
        cudaFree(g);
        cudaFree(m);
        cudaFree(v);
        cudaFree(loss);
        cudaFree(wb);
    }
};

#define MTRY(expr)                                                                          \
    do {                                                                                    \
        cudaError_t _e = (expr);                                                            \
        if (_e != cudaSuccess) return mfail(LSG_E_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
    } while (0)

static int mlp_prepare_kernels(int F) {
    size_t b = smem_bytes(F);
    MTRY(cudaFuncSetAttribute(k_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b));
    MTRY(cudaFuncSetAttribute(k_backward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b));
    return 0;
}

extern "C" {

const char* lsg_mlp_last_error(void) { return g_mlp_err.c_str(); }

int lsg_mlp_create(int32_t n_features, const float* params, lsg_mlp** out) {
    if (!out || !params || n_features < 1 || n_features > MAXF) return mfail(LSG_E_INVALID, "bad MLP arguments");
    lsg_mlp* m = new lsg_mlp();
    m->F = n_features;
    m->np = Layout(n_features).total;
    size_t b = m->np * sizeof(float);
    if (cudaMalloc(&m->p, b) || cudaMalloc(&m->g, b) || cudaMalloc(&m->m, b) || cudaMalloc(&m->v, b) ||
        cudaMalloc(&m->loss, sizeof(float)) || cudaMalloc(&m->wb, m->np * sizeof(__nv_bfloat16))) {
        delete m;
        return mfail(LSG_E_CUDA, "cudaMalloc failed for the MLP");
    }
    cudaMemcpy(m->p, params, b, cudaMemcpyHostToDevice);
    cudaMemset(m->m, 0, b);
    cudaMemset(m->v, 0, b);
    k_to_bf16<<<(unsigned)((m->np + 255) / 256), 256>>>(m->p, m->np, m->wb);
    int rc = mlp_prepare_kernels(n_features);
    if (rc) { delete m; return rc; }
    MTRY(cudaDeviceSynchronize());
    *out = m;
    return 0;
}

void lsg_mlp_destroy(lsg_mlp* m) { delete m; }

int64_t lsg_mlp_num_params(int32_t n_features) { return Layout(n_features).total; }

int lsg_mlp_get_params(const lsg_mlp* m, float* params) {
    if (!m || !params) return mfail(LSG_E_INVALID, "null argument");
    MTRY(cudaMemcpy(params, m->p, m->np * sizeof(float), cudaMemcpyDeviceToHost));
    return 0;
}

int lsg_mlp_forward(lsg_mlp* m, const float* X, int64_t rows, float* out, void* stream) {
    if (!m || !X || !out || rows < 0) return mfail(LSG_E_INVALID, "bad argument");
    if (rows == 0) return 0;
    int64_t tiles = (rows + TR - 1) / TR;
    unsigned grid = (unsigned)(tiles < 2048 ? tiles : 2048);
    k_forward<<<grid, 256, smem_bytes(m->F), (cudaStream_t)stream>>>(m->wb, m->p, X, rows, m->F, out);
    MTRY(cudaGetLastError());
    return 0;
}

int lsg_mlp_gradient(lsg_mlp* m, const float* X, const float* Y, int64_t rows, float* grad_host, float* loss_host) {
    if (!m || !X || !Y || rows < 1) return mfail(LSG_E_INVALID, "bad argument");
    MTRY(cudaMemset(m->g, 0, m->np * sizeof(float)));
    MTRY(cudaMemset(m->loss, 0, sizeof(float)));
    int64_t tiles = (rows + TR - 1) / TR;
    unsigned grid = (unsigned)(tiles < 592 ? tiles : 592);
    k_backward<<<grid, 256, smem_bytes(m->F)>>>(m->wb, m->p, X, Y, rows, m->F, m->g, m->loss);
    MTRY(cudaGetLastError());
    if (grad_host) MTRY(cudaMemcpy(grad_host, m->g, m->np * sizeof(float), cudaMemcpyDeviceToHost));
    if (loss_host) {
        float l;
        MTRY(cudaMemcpy(&l, m->loss, sizeof(float), cudaMemcpyDeviceToHost));
        *loss_host = l / (float)rows;
    }
    return 0;
}

int lsg_mlp_train_step(lsg_mlp* m, const float* X, const float* Y, int64_t rows, float lr, float* loss_host) {
    int rc = lsg_mlp_gradient(m, X, Y, rows, nullptr, loss_host);
    if (rc) return rc;
    m->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    float c1 = 1.f - powf(b1, (float)m->step), c2 = 1.f - powf(b2, (float)m->step);
    k_adam<<<(unsigned)((m->np + 255) / 256), 256>>>(m->p, m->g, m->m, m->v, m->np, lr, b1, b2, 1e-8f, c1, c2, m->wb);
    MTRY(cudaGetLastError());
    return 0;
}

}  // extern "C"
