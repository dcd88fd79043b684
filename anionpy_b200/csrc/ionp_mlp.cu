// The schedule picker's network: a 3-layer perceptron (FP32, ReLU hidden
// layers) that maps a call's features to a predicted log-time for each of the
// 48 schedules, with hand-written forward, backward and Adam kernels. No
// counterpart in the reference. Dimensions are tiny (inputs ~30, width 64,
// 48 outputs), so every kernel is a plain thread-per-output loop with a fixed
// summation order: training is deterministic run to run.
//
// Parameter layout (one flat float buffer): W1[nin][h], b1[h], W2[h][h], b2[h],
// W3[h][nout], b3[nout]; W[k][n] multiplies input k into output n.
#include <cmath>
#include <cstring>
#include <vector>
#include "ionp_host.h"
#include "ionp_internal.h"

namespace ionp {
namespace {

constexpr int MLP_THREADS = 256;

// Y[b][n] = act(sum_k X[b][k] W[k][n] + bias[n])
__global__ void __launch_bounds__(MLP_THREADS) k_dense_fwd(const float* __restrict__ X, const float* __restrict__ W,
                                                           const float* __restrict__ bias, float* __restrict__ Y,
                                                           int B, int K, int N, int relu) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B * N) return;
    const int b = i / N, n = i - b * N;
    float acc = bias[n];
    const float* x = X + (size_t)b * K;
    for (int k = 0; k < K; ++k) acc = __fmaf_rn(x[k], W[(size_t)k * N + n], acc);
    Y[i] = relu ? fmaxf(acc, 0.0f) : acc;
}

// dY = 2 (Y - T) / (B * N) over the entries with mask 1; loss partial sums
// per block (the host adds them in block order).
__global__ void __launch_bounds__(MLP_THREADS) k_mse(const float* __restrict__ Y, const float* __restrict__ T,
                                                     const float* __restrict__ M, float* __restrict__ dY,
                                                     float* __restrict__ loss_blocks, int count, float scale) {
    __shared__ float red[MLP_THREADS];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.0f;
    if (i < count) {
        const float m = M ? M[i] : 1.0f;
        const float d = (Y[i] - T[i]) * m;
        dY[i] = 2.0f * d * scale;
        l = d * d * scale;
    }
    red[threadIdx.x] = l;
    __syncthreads();
    for (int s = MLP_THREADS / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) loss_blocks[blockIdx.x] = red[0];
}

// dX[b][k] = (sum_n dY[b][n] W[k][n]) * (H[b][k] > 0)   (H = the ReLU output)
__global__ void __launch_bounds__(MLP_THREADS) k_dense_bwd_in(const float* __restrict__ dY, const float* __restrict__ W,
                                                              const float* __restrict__ H, float* __restrict__ dX,
                                                              int B, int K, int N) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B * K) return;
    const int b = i / K, k = i - b * K;
    float acc = 0.0f;
    const float* dy = dY + (size_t)b * N;
    const float* w = W + (size_t)k * N;
    for (int n = 0; n < N; ++n) acc = __fmaf_rn(dy[n], w[n], acc);
    dX[i] = H[i] > 0.0f ? acc : 0.0f;
}

// dW[k][n] = sum_b X[b][k] dY[b][n];  db[n] = sum_b dY[b][n]   (b ascending)
__global__ void __launch_bounds__(MLP_THREADS) k_dense_bwd_w(const float* __restrict__ X, const float* __restrict__ dY,
                                                             float* __restrict__ dW, float* __restrict__ db, int B, int K,
                                                             int N) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < K * N) {
        const int k = i / N, n = i - k * N;
        float acc = 0.0f;
        for (int b = 0; b < B; ++b) acc = __fmaf_rn(X[(size_t)b * K + k], dY[(size_t)b * N + n], acc);
        dW[i] = acc;
    } else if (i < K * N + N) {
        const int n = i - K * N;
        float acc = 0.0f;
        for (int b = 0; b < B; ++b) acc += dY[(size_t)b * N + n];
        db[n] = acc;
    }
}

__global__ void __launch_bounds__(MLP_THREADS) k_adam(float* __restrict__ p, const float* __restrict__ g,
                                                      float* __restrict__ m, float* __restrict__ v, int n, float lr,
                                                      float b1, float b2, float eps, float c1, float c2, float wd) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i] + wd * p[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float mh = mi / c1, vh = vi / c2;
    p[i] -= lr * mh / (sqrtf(vh) + eps);
}

int blocks(int n) { return (n + MLP_THREADS - 1) / MLP_THREADS; }

}  // namespace
}  // namespace ionp

using namespace ionp;

struct IonpMlp {
    int nin = 0, h = 0, nout = 0;
    size_t nparam = 0;
    float* p = nullptr;   // parameters
    float* g = nullptr;   // gradients
    float* m = nullptr;   // Adam moments
    float* v = nullptr;
    int64_t step = 0;
    // activations / gradients for the largest batch seen
    int cap = 0;
    float *h1 = nullptr, *h2 = nullptr, *y = nullptr, *d3 = nullptr, *d2 = nullptr, *d1 = nullptr, *lossb = nullptr;
    std::vector<float> lossh;
};

namespace {
size_t off_w1(const IonpMlp* m) { return 0; }
size_t off_b1(const IonpMlp* m) { return (size_t)m->nin * m->h; }
size_t off_w2(const IonpMlp* m) { return off_b1(m) + m->h; }
size_t off_b2(const IonpMlp* m) { return off_w2(m) + (size_t)m->h * m->h; }
size_t off_w3(const IonpMlp* m) { return off_b2(m) + m->h; }
size_t off_b3(const IonpMlp* m) { return off_w3(m) + (size_t)m->h * m->nout; }

void free_acts(IonpMlp* m) {
    float** bufs[] = {&m->h1, &m->h2, &m->y, &m->d3, &m->d2, &m->d1, &m->lossb};
    for (float** b : bufs) {
        if (*b) scratch_free(*b, nullptr);
        *b = nullptr;
    }
    m->cap = 0;
}

int32_t ensure_acts(IonpMlp* m, int B) {
    if (B <= m->cap) return IONP_OK;
    free_acts(m);
    const size_t hb = (size_t)B * m->h * 4, ob = (size_t)B * m->nout * 4;
    m->h1 = (float*)scratch_alloc(hb, nullptr);
    m->h2 = (float*)scratch_alloc(hb, nullptr);
    m->y = (float*)scratch_alloc(ob, nullptr);
    m->d3 = (float*)scratch_alloc(ob, nullptr);
    m->d2 = (float*)scratch_alloc(hb, nullptr);
    m->d1 = (float*)scratch_alloc(hb, nullptr);
    m->lossb = (float*)scratch_alloc((size_t)blocks(B * m->nout) * 4 + 16, nullptr);
    if (!m->h1 || !m->h2 || !m->y || !m->d3 || !m->d2 || !m->d1 || !m->lossb) {
        free_acts(m);
        return IONP_ERR_OOM;
    }
    m->cap = B;
    return IONP_OK;
}

void forward(IonpMlp* m, const float* x, int B, float* y, cudaStream_t s) {
    k_dense_fwd<<<blocks(B * m->h), MLP_THREADS, 0, s>>>(x, m->p + off_w1(m), m->p + off_b1(m), m->h1, B, m->nin, m->h, 1);
    k_dense_fwd<<<blocks(B * m->h), MLP_THREADS, 0, s>>>(m->h1, m->p + off_w2(m), m->p + off_b2(m), m->h2, B, m->h, m->h, 1);
    k_dense_fwd<<<blocks(B * m->nout), MLP_THREADS, 0, s>>>(m->h2, m->p + off_w3(m), m->p + off_b3(m), y, B, m->h, m->nout, 0);
    count_launch(3);
}

// fills m->g with d(loss)/d(params) for the batch; returns the loss
int32_t gradients(IonpMlp* m, const float* x, const float* t, const float* mask, int B, float* loss, cudaStream_t s) {
    int32_t st = ensure_acts(m, B);
    if (st) return st;
    forward(m, x, B, m->y, s);
    const int cnt = B * m->nout;
    k_mse<<<blocks(cnt), MLP_THREADS, 0, s>>>(m->y, t, mask, m->d3, m->lossb, cnt, 1.0f / (float)cnt);
    k_dense_bwd_w<<<blocks(m->h * m->nout + m->nout), MLP_THREADS, 0, s>>>(m->h2, m->d3, m->g + off_w3(m), m->g + off_b3(m), B,
                                                                           m->h, m->nout);
    k_dense_bwd_in<<<blocks(B * m->h), MLP_THREADS, 0, s>>>(m->d3, m->p + off_w3(m), m->h2, m->d2, B, m->h, m->nout);
    k_dense_bwd_w<<<blocks(m->h * m->h + m->h), MLP_THREADS, 0, s>>>(m->h1, m->d2, m->g + off_w2(m), m->g + off_b2(m), B, m->h,
                                                                     m->h);
    k_dense_bwd_in<<<blocks(B * m->h), MLP_THREADS, 0, s>>>(m->d2, m->p + off_w2(m), m->h1, m->d1, B, m->h, m->h);
    k_dense_bwd_w<<<blocks(m->nin * m->h + m->h), MLP_THREADS, 0, s>>>(x, m->d1, m->g + off_w1(m), m->g + off_b1(m), B, m->nin,
                                                                       m->h);
    count_launch(6);
    if (loss) {
        const int nb = blocks(cnt);
        m->lossh.resize(nb);
        st = cuda_err(cudaMemcpyAsync(m->lossh.data(), m->lossb, (size_t)nb * 4, cudaMemcpyDeviceToHost, s), "mlp loss");
        if (!st) st = cuda_err(cudaStreamSynchronize(s), "mlp loss");
        if (st) return st;
        double acc = 0;
        for (float f : m->lossh) acc += f;
        *loss = (float)acc;
    }
    return cuda_err(cudaGetLastError(), "mlp backward");
}

}  // namespace

extern "C" {

int32_t ionp_mlp_create(IonpMlp** out, int32_t nin, int32_t hidden, int32_t nout, uint64_t seed) {
    if (!out || nin <= 0 || hidden <= 0 || nout <= 0) return set_err(IONP_ERR_INVALID, "bad network shape");
    IonpMlp* m = new IonpMlp();
    m->nin = nin; m->h = hidden; m->nout = nout;
    m->nparam = off_b3(m) + nout;
    const size_t bytes = m->nparam * 4;
    m->p = (float*)scratch_alloc(bytes, nullptr);
    m->g = (float*)scratch_alloc(bytes, nullptr);
    m->m = (float*)scratch_alloc(bytes, nullptr);
    m->v = (float*)scratch_alloc(bytes, nullptr);
    if (!m->p || !m->g || !m->m || !m->v) { delete m; return IONP_ERR_OOM; }
    // He-uniform initialisation from a seeded xorshift on the host
    std::vector<float> init(m->nparam, 0.0f);
    uint64_t x = seed * 0x9E3779B97F4A7C15ull + 1;
    auto uni = [&]() {
        x ^= x << 13; x ^= x >> 7; x ^= x << 17;
        return (double)(x >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
    };
    auto fill = [&](size_t off, int fan_in, size_t n) {
        const double lim = std::sqrt(6.0 / fan_in);
        for (size_t i = 0; i < n; ++i) init[off + i] = (float)(uni() * lim);
    };
    fill(off_w1(m), nin, (size_t)nin * hidden);
    fill(off_w2(m), hidden, (size_t)hidden * hidden);
    fill(off_w3(m), hidden, (size_t)hidden * nout);
    int32_t st = cuda_err(cudaMemcpy(m->p, init.data(), bytes, cudaMemcpyHostToDevice), "mlp init");
    if (!st) st = cuda_err(cudaMemset(m->m, 0, bytes), "mlp init");
    if (!st) st = cuda_err(cudaMemset(m->v, 0, bytes), "mlp init");
    if (!st) st = cuda_err(cudaMemset(m->g, 0, bytes), "mlp init");
    if (st) { delete m; return st; }
    *out = m;
    return IONP_OK;
}

int32_t ionp_mlp_destroy(IonpMlp* m) {
    if (!m) return IONP_OK;
    cudaDeviceSynchronize();
    free_acts(m);
    scratch_free(m->p, nullptr);
    scratch_free(m->g, nullptr);
    scratch_free(m->m, nullptr);
    scratch_free(m->v, nullptr);
    delete m;
    return IONP_OK;
}

int32_t ionp_mlp_num_params(IonpMlp* m, int64_t* n) {
    if (!m || !n) return set_err(IONP_ERR_INVALID, "bad arguments");
    *n = (int64_t)m->nparam;
    return IONP_OK;
}

/* which = 0 parameters, 1 gradients of the last ionp_mlp_gradients/step */
int32_t ionp_mlp_get(IonpMlp* m, int32_t which, float* host, int64_t n) {
    if (!m || !host || n != (int64_t)m->nparam) return set_err(IONP_ERR_INVALID, "bad arguments");
    return cuda_err(cudaMemcpy(host, which ? m->g : m->p, (size_t)n * 4, cudaMemcpyDeviceToHost), "mlp get");
}

int32_t ionp_mlp_set_params(IonpMlp* m, const float* host, int64_t n) {
    if (!m || !host || n != (int64_t)m->nparam) return set_err(IONP_ERR_INVALID, "bad arguments");
    m->step = 0;
    int32_t st = cuda_err(cudaMemcpy(m->p, host, (size_t)n * 4, cudaMemcpyHostToDevice), "mlp set");
    if (!st) st = cuda_err(cudaMemset(m->m, 0, (size_t)n * 4), "mlp set");
    if (!st) st = cuda_err(cudaMemset(m->v, 0, (size_t)n * 4), "mlp set");
    return st;
}

int32_t ionp_mlp_forward(IonpMlp* m, const float* x, int32_t batch, float* y, IonpStream stream) {
    if (!m || !x || !y || batch <= 0) return set_err(IONP_ERR_INVALID, "bad arguments");
    int32_t st = ensure_acts(m, batch);
    if (st) return st;
    forward(m, x, batch, y, (cudaStream_t)stream);
    return cuda_err(cudaGetLastError(), "mlp forward");
}

int32_t ionp_mlp_gradients(IonpMlp* m, const float* x, const float* t, const float* mask, int32_t batch, float* loss,
                           IonpStream stream) {
    if (!m || !x || !t || batch <= 0) return set_err(IONP_ERR_INVALID, "bad arguments");
    return gradients(m, x, t, mask, batch, loss, (cudaStream_t)stream);
}

int32_t ionp_mlp_train_step(IonpMlp* m, const float* x, const float* t, const float* mask, int32_t batch, float lr,
                            float weight_decay, float* loss, IonpStream stream) {
    if (!m || !x || !t || batch <= 0) return set_err(IONP_ERR_INVALID, "bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    int32_t st = gradients(m, x, t, mask, batch, loss, s);
    if (st) return st;
    m->step++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - (float)std::pow((double)b1, (double)m->step);
    const float c2 = 1.0f - (float)std::pow((double)b2, (double)m->step);
    k_adam<<<blocks((int)m->nparam), MLP_THREADS, 0, s>>>(m->p, m->g, m->m, m->v, (int)m->nparam, lr, b1, b2, 1e-8f, c1, c2,
                                                         weight_decay);
    count_launch();
    return cuda_err(cudaGetLastError(), "mlp adam");
}

}  // extern "C"
