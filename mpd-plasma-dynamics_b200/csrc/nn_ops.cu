// Element-wise and reduction kernels of the surrogate network (FP32), around
// the tensor-core GEMM of nn_gemm.cu: bias + activation, its derivative,
// column sums (bias gradients), sums of split-K partial products, the
// squared-error loss and its gradient, and the Adam update.  All sums are
// deterministic (fixed partition, fixed order).
#include <cuda_runtime.h>

#include <cmath>
#include <string>

#include "../../include/mpd_b200.h"

namespace mpd {
void SetLastError(const std::string &msg);
}

namespace {

constexpr int kThreads = 256;

int Launched(const char *what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        mpd::SetLastError(std::string(what) + ": " + cudaGetErrorString(e));
        return MPD_ERR_CUDA;
    }
    return MPD_OK;
}

int Blocks(long long n) {
    long long b = (n + kThreads - 1) / kThreads;
    if (b > 148 * 32) b = 148 * 32;
    return (int)(b > 0 ? b : 1);
}

// GELU, tanh form: 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))).
__device__ __forceinline__ float gelu(float x, float &dgelu) {
    const float c = 0.7978845608028654f;  // sqrt(2 / pi)
    const float u = c * (x + 0.044715f * x * x * x);
    const float t = tanhf(u);
    dgelu = 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * c * (1.0f + 3.0f * 0.044715f * x * x);
    return 0.5f * x * (1.0f + t);
}

// z[r][c] += bias[c]; out[r][c] = act ? gelu(z) : z.
__global__ void bias_act_kernel(float *z, const float *bias, float *out, long long rows, int cols,
                                int act) {
    const long long n = rows * cols;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float v = z[i] + (bias ? bias[i % cols] : 0.0f);
        z[i] = v;
        float d;
        out[i] = act ? gelu(v, d) : v;
    }
}

// g_z = g_out * gelu'(z)
__global__ void act_bwd_kernel(const float *g_out, const float *z, float *g_z, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        float d;
        gelu(z[i], d);
        g_z[i] = g_out[i] * d;
    }
}

// Column sums in two fixed-order stages: block (bx, by) sums rows
// by, by + kColSlices, ... of 32 columns into work[by][c]; then one thread
// per column adds the kColSlices partials in order.
constexpr int kColSlices = 128;

__global__ void colsum_partial_kernel(const float *x, long long rows, int cols, float *work) {
    __shared__ float part[8][33];
    const int c = blockIdx.x * 32 + (threadIdx.x & 31);
    const int ry = threadIdx.x >> 5;
    float s = 0.0f;
    if (c < cols)
        for (long long r = (long long)blockIdx.y * 8 + ry; r < rows; r += 8LL * kColSlices)
            s += x[r * cols + c];
    part[ry][threadIdx.x & 31] = s;
    __syncthreads();
    if (ry == 0 && c < cols) {
        float t = 0.0f;
        for (int k = 0; k < 8; ++k) t += part[k][threadIdx.x & 31];
        work[(size_t)blockIdx.y * cols + c] = t;
    }
}

__global__ void colsum_final_kernel(const float *work, int cols, float *out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float t = 0.0f;
    for (int k = 0; k < kColSlices; ++k) t += work[(size_t)k * cols + c];
    out[c] = t;
}

// out[i] = (accumulate ? out[i] : 0) + sum_t parts[t][i]
__global__ void sum_parts_kernel(const float *parts, int nparts, long long n, float *out,
                                 int accumulate) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        float s = accumulate ? out[i] : 0.0f;
        for (int t = 0; t < nparts; ++t) s += parts[(long long)t * n + i];
        out[i] = s;
    }
}

// grad = 2 (pred - target) / n; per-block partial sums of the squared error.
__global__ void mse_kernel(const float *pred, const float *target, long long n, float *grad,
                           double *partial) {
    __shared__ double red[kThreads];
    double s = 0.0;
    const float inv = 2.0f / (float)n;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float d = pred[i] - target[i];
        s += (double)d * d;
        if (grad) grad[i] = inv * d;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = kThreads / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// One block: thread t sums partials t, t + 256, ... in order, then a fixed tree.
__global__ void sum_partials_kernel(const double *partial, int n, double scale, double *out) {
    __shared__ double red[kThreads];
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += kThreads) s += partial[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = kThreads / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0] * scale;
}

// Adam: m = b1 m + (1-b1) g; v = b2 v + (1-b2) g^2;
// p -= lr (m / (1-b1^t)) / (sqrt(v / (1-b2^t)) + eps)
__global__ void adam_kernel(float *p, const float *g, float *m, float *v, long long n, float lr,
                            float b1, float b2, float eps, float c1, float c2) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

}  // namespace

extern "C" {

int mpd_nn_bias_act(float *z, const float *bias, float *out, long long rows, int cols, int act,
                    void *stream) {
    if (!z || !out || rows < 0 || cols <= 0) {
        mpd::SetLastError("mpd_nn_bias_act: bad arguments");
        return MPD_ERR_INVALID;
    }
    bias_act_kernel<<<Blocks(rows * cols), kThreads, 0, (cudaStream_t)stream>>>(z, bias, out, rows,
                                                                                cols, act);
    return Launched("mpd_nn_bias_act");
}

int mpd_nn_act_bwd(const float *g_out, const float *z, float *g_z, long long n, void *stream) {
    if (!g_out || !z || !g_z || n < 0) {
        mpd::SetLastError("mpd_nn_act_bwd: bad arguments");
        return MPD_ERR_INVALID;
    }
    act_bwd_kernel<<<Blocks(n), kThreads, 0, (cudaStream_t)stream>>>(g_out, z, g_z, n);
    return Launched("mpd_nn_act_bwd");
}

int mpd_nn_colsum(const float *x, long long rows, int cols, float *out, float *work,
                  void *stream) {
    if (!x || !out || !work || rows < 0 || cols <= 0) {
        mpd::SetLastError("mpd_nn_colsum: bad arguments");
        return MPD_ERR_INVALID;
    }
    colsum_partial_kernel<<<dim3((cols + 31) / 32, kColSlices), kThreads, 0,
                            (cudaStream_t)stream>>>(x, rows, cols, work);
    colsum_final_kernel<<<(cols + 127) / 128, 128, 0, (cudaStream_t)stream>>>(work, cols, out);
    return Launched("mpd_nn_colsum");
}

int mpd_nn_sum_parts(const float *parts, int nparts, long long n, float *out, int accumulate,
                     void *stream) {
    if (!parts || !out || nparts < 1 || n < 0) {
        mpd::SetLastError("mpd_nn_sum_parts: bad arguments");
        return MPD_ERR_INVALID;
    }
    sum_parts_kernel<<<Blocks(n), kThreads, 0, (cudaStream_t)stream>>>(parts, nparts, n, out,
                                                                       accumulate);
    return Launched("mpd_nn_sum_parts");
}

/* partial: at least 148 * 32 doubles of scratch; loss: one double (mean
 * squared error over the n values). */
int mpd_nn_mse(const float *pred, const float *target, long long n, float *grad, double *partial,
               double *loss, void *stream) {
    if (!pred || !target || !partial || !loss || n <= 0) {
        mpd::SetLastError("mpd_nn_mse: bad arguments");
        return MPD_ERR_INVALID;
    }
    const int nb = Blocks(n);
    mse_kernel<<<nb, kThreads, 0, (cudaStream_t)stream>>>(pred, target, n, grad, partial);
    sum_partials_kernel<<<1, kThreads, 0, (cudaStream_t)stream>>>(partial, nb, 1.0 / (double)n,
                                                                 loss);
    return Launched("mpd_nn_mse");
}

int mpd_nn_adam(float *p, const float *g, float *m, float *v, long long n, float lr, float b1,
                float b2, float eps, int step, void *stream) {
    if (!p || !g || !m || !v || n < 0 || step < 1) {
        mpd::SetLastError("mpd_nn_adam: bad arguments");
        return MPD_ERR_INVALID;
    }
    const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    adam_kernel<<<Blocks(n), kThreads, 0, (cudaStream_t)stream>>>(p, g, m, v, n, lr, b1, b2, eps,
                                                                  c1, c2);
    return Launched("mpd_nn_adam");
}

}  // extern "C"
