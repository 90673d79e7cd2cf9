// The learned warm start's network: a small fully connected MLP (GELU hidden layers,
// linear output) trained in FP32 on the device with hand-written forward, backward and
// Adam kernels. It maps (composition, temperature) to the zero-pressure lattice constant
// and initial C11, C12, C44, so that a production run can start near equilibrium.
//
// Sizes are small (inputs and widths of tens, a few thousand samples), so every kernel is a
// plain FP32 FMA loop with one thread per output element and sums in a fixed order: no
// atomics, training is bit-for-bit repeatable. A training step (forward, loss, backward,
// Adam) is captured once as a CUDA graph and replayed.
//
// Parameter layout (also of gradients and of the host copies): for each layer l in order,
// W_l as in_l x out_l row-major (W[i * out + o]), then b_l (out_l).
#include <cuda_runtime.h>

#include <cmath>
#include <algorithm>
#include <cstring>
#include <random>
#include <vector>

#include "host_tables.h"
#include "mdelast.h"

using mdelast::clear_error;
using mdelast::fail;

namespace {

constexpr int kT = 256;

__device__ __forceinline__ float gelu(float z) {
    return 0.5f * z * (1.f + erff(z * 0.70710678118654752f));
}
__device__ __forceinline__ float gelu_d(float z) {
    // d/dz [z Phi(z)] = Phi(z) + z phi(z)
    return 0.5f * (1.f + erff(z * 0.70710678118654752f)) +
           z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// Z = X W + b; A = gelu(Z) for hidden layers, A = Z for the output layer
__global__ void k_fwd(const float *X, const float *W, const float *b, float *Z, float *A, int n,
                      int in, int out, int act) {
    int const k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n * out)
        return;
    int const s = k / out, o = k % out;
    float z = b[o];
    for (int i = 0; i < in; ++i)
        z = fmaf(X[s * in + i], W[i * out + o], z);
    Z[k] = z;
    A[k] = act ? gelu(z) : z;
}

// mean-squared error over n x out outputs: dY = 2 (Y - T) / (n out), loss in one block with
// a fixed-order tree
__global__ void k_loss(const float *Y, const float *Tg, float *dY, float *loss, int m) {
    __shared__ float part[kT];
    float const inv = 1.f / static_cast<float>(m);
    float acc = 0.f;
    for (int k = threadIdx.x; k < m; k += kT) {
        float const d = Y[k] - Tg[k];
        dY[k] = 2.f * d * inv;
        acc = fmaf(d, d, acc);
    }
    part[threadIdx.x] = acc;
    __syncthreads();
    for (int w = kT / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            part[threadIdx.x] += part[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        *loss = part[0] * inv;
}

// dZ = dA * gelu'(Z)
__global__ void k_bwd_act(const float *dA, const float *Z, float *dZ, int m) {
    int const k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < m)
        dZ[k] = dA[k] * gelu_d(Z[k]);
}

// dX = dZ W^T
__global__ void k_bwd_dx(const float *dZ, const float *W, float *dX, int n, int in, int out) {
    int const k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n * in)
        return;
    int const s = k / in, i = k % in;
    float acc = 0.f;
    for (int o = 0; o < out; ++o)
        acc = fmaf(dZ[s * out + o], W[i * out + o], acc);
    dX[k] = acc;
}

// dW = X^T dZ, db = column sums of dZ (thread per parameter, samples in order)
__global__ void k_bwd_dw(const float *X, const float *dZ, float *dW, float *db, int n, int in,
                         int out) {
    int const k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < in * out) {
        int const i = k / out, o = k % out;
        float acc = 0.f;
        for (int s = 0; s < n; ++s)
            acc = fmaf(X[s * in + i], dZ[s * out + o], acc);
        dW[k] = acc;
    } else if (k < in * out + out) {
        int const o = k - in * out;
        float acc = 0.f;
        for (int s = 0; s < n; ++s)
            acc += dZ[s * out + o];
        db[o] = acc;
    }
}

// Adam (Kingma & Ba 2015) with bias correction; the step count lives on the device so that
// a captured graph can be replayed
__global__ void k_adam(float *p, const float *g, float *m1, float *m2, int np, float lr,
                       const int *t) {
    int const k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= np)
        return;
    float const b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    float const step = static_cast<float>(*t + 1);
    float const c1 = 1.f - powf(b1, step), c2 = 1.f - powf(b2, step);
    float const gk = g[k];
    float const a = b1 * m1[k] + (1.f - b1) * gk;
    float const v = b2 * m2[k] + (1.f - b2) * gk * gk;
    m1[k] = a;
    m2[k] = v;
    p[k] -= lr * (a / c1) / (sqrtf(v / c2) + eps);
}

__global__ void k_step_inc(int *t) {
    if (threadIdx.x == 0 && blockIdx.x == 0)
        *t += 1;
}

unsigned blocks(long m) { return static_cast<unsigned>((m + kT - 1) / kT); }

} // namespace

#define MCK(call)                                                                              \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return fail(MDELAST_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_));            \
    } while (0)

struct mdelast_mlp_s {
    int device = 0;
    int L = 0;                  // layers
    std::vector<int> w;         // widths, L + 1
    std::vector<long> off_w, off_b;
    long np = 0;
    cudaStream_t stream = nullptr;
    float *p = nullptr, *g = nullptr, *m1 = nullptr, *m2 = nullptr;
    int *t = nullptr;
    // activations for a batch of cap samples: per layer Z and A; A[0] is the input
    int cap = 0;
    std::vector<float *> Z, A, dA;
    float *Yt = nullptr, *dZ = nullptr, *loss = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_n = -1;
    float graph_lr = 0.f;

    ~mdelast_mlp_s() {
        cudaSetDevice(device);
        if (graph)
            cudaGraphExecDestroy(graph);
        for (float *q : {p, g, m1, m2, Yt, dZ, loss})
            cudaFree(q);
        cudaFree(t);
        for (auto *v : {&Z, &A, &dA})
            for (float *q : *v)
                cudaFree(q);
        if (stream)
            cudaStreamDestroy(stream);
    }

    int reserve(int n) {
        if (n <= cap)
            return MDELAST_OK;
        if (graph) {
            cudaGraphExecDestroy(graph);
            graph = nullptr;
            graph_n = -1;
        }
        for (auto *v : {&Z, &A, &dA})
            for (float *&q : *v) {
                cudaFree(q);
                q = nullptr;
            }
        cudaFree(Yt);
        cudaFree(dZ);
        Z.assign(L + 1, nullptr);
        A.assign(L + 1, nullptr);
        dA.assign(L + 1, nullptr);
        int wmax = 0;
        for (int k = 0; k <= L; ++k) {
            MCK(cudaMalloc(&A[k], sizeof(float) * static_cast<size_t>(n) * w[k]));
            MCK(cudaMalloc(&dA[k], sizeof(float) * static_cast<size_t>(n) * w[k]));
            if (k > 0)
                MCK(cudaMalloc(&Z[k], sizeof(float) * static_cast<size_t>(n) * w[k]));
            wmax = std::max(wmax, w[k]);
        }
        MCK(cudaMalloc(&Yt, sizeof(float) * static_cast<size_t>(n) * w[L]));
        MCK(cudaMalloc(&dZ, sizeof(float) * static_cast<size_t>(n) * wmax));
        cap = n;
        return MDELAST_OK;
    }

    void forward(int n, cudaStream_t s) {
        for (int l = 0; l < L; ++l)
            k_fwd<<<blocks(static_cast<long>(n) * w[l + 1]), kT, 0, s>>>(
                A[l], p + off_w[l], p + off_b[l], Z[l + 1], A[l + 1], n, w[l], w[l + 1],
                l + 1 < L);
    }

    // gradients of the mean-squared error of A[L] against Yt into g
    void backward(int n, cudaStream_t s) {
        k_loss<<<1, kT, 0, s>>>(A[L], Yt, dA[L], loss, n * w[L]);
        for (int l = L - 1; l >= 0; --l) {
            long const m = static_cast<long>(n) * w[l + 1];
            const float *dz = dA[l + 1];
            if (l + 1 < L) {
                k_bwd_act<<<blocks(m), kT, 0, s>>>(dA[l + 1], Z[l + 1], dZ, static_cast<int>(m));
                dz = dZ;
            }
            k_bwd_dw<<<blocks(static_cast<long>(w[l]) * w[l + 1] + w[l + 1]), kT, 0, s>>>(
                A[l], dz, g + off_w[l], g + off_b[l], n, w[l], w[l + 1]);
            if (l > 0)
                k_bwd_dx<<<blocks(static_cast<long>(n) * w[l]), kT, 0, s>>>(
                    dz, p + off_w[l], dA[l], n, w[l], w[l + 1]);
        }
    }

    int upload(const float *x, const float *y, int n) {
        if (int rc = reserve(n))
            return rc;
        MCK(cudaMemcpyAsync(A[0], x, sizeof(float) * static_cast<size_t>(n) * w[0],
                            cudaMemcpyHostToDevice, stream));
        if (y)
            MCK(cudaMemcpyAsync(Yt, y, sizeof(float) * static_cast<size_t>(n) * w[L],
                                cudaMemcpyHostToDevice, stream));
        return MDELAST_OK;
    }
};

extern "C" {

int mdelast_mlp_create(int32_t n_layers, const int32_t *widths, uint64_t seed, int32_t device,
                       mdelast_mlp **out) {
    clear_error();
    if (!widths || !out || n_layers < 1 || n_layers > MDELAST_MLP_MAX_LAYERS)
        return fail(MDELAST_ERR_ARGUMENT, "an MLP needs 1..%d layers", MDELAST_MLP_MAX_LAYERS);
    for (int k = 0; k <= n_layers; ++k)
        if (widths[k] < 1 || widths[k] > 4096)
            return fail(MDELAST_ERR_ARGUMENT, "layer width %d out of range", widths[k]);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(MDELAST_ERR_NO_DEVICE, "no CUDA device: the MLP kernels need one");
    }
    if (device < 0 || device >= ndev)
        return fail(MDELAST_ERR_ARGUMENT, "device %d not present", device);
    MCK(cudaSetDevice(device));
    auto *m = new mdelast_mlp_s();
    m->device = device;
    m->L = n_layers;
    m->w.assign(widths, widths + n_layers + 1);
    for (int l = 0; l < n_layers; ++l) {
        m->off_w.push_back(m->np);
        m->np += static_cast<long>(m->w[l]) * m->w[l + 1];
        m->off_b.push_back(m->np);
        m->np += m->w[l + 1];
    }
    // Glorot-normal weights, zero biases, from a 64-bit Mersenne Twister seeded by `seed`
    std::vector<float> h(static_cast<size_t>(m->np), 0.f);
    std::mt19937_64 rng(seed);
    for (int l = 0; l < n_layers; ++l) {
        std::normal_distribution<double> nd(0., std::sqrt(2. / (m->w[l] + m->w[l + 1])));
        for (long k = 0; k < static_cast<long>(m->w[l]) * m->w[l + 1]; ++k)
            h[static_cast<size_t>(m->off_w[l] + k)] = static_cast<float>(nd(rng));
    }
    size_t const bytes = sizeof(float) * static_cast<size_t>(m->np);
    cudaError_t e = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking);
    for (float **q : {&m->p, &m->g, &m->m1, &m->m2})
        if (e == cudaSuccess)
            e = cudaMalloc(q, bytes);
    if (e == cudaSuccess)
        e = cudaMalloc(&m->t, sizeof(int));
    if (e == cudaSuccess)
        e = cudaMalloc(&m->loss, sizeof(float));
    if (e == cudaSuccess)
        e = cudaMemcpy(m->p, h.data(), bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemset(m->m1, 0, bytes);
    if (e == cudaSuccess)
        e = cudaMemset(m->m2, 0, bytes);
    if (e == cudaSuccess)
        e = cudaMemset(m->g, 0, bytes);
    if (e == cudaSuccess)
        e = cudaMemset(m->t, 0, sizeof(int));
    if (e != cudaSuccess) {
        delete m;
        return fail(MDELAST_ERR_CUDA, "MLP set-up: %s", cudaGetErrorString(e));
    }
    *out = m;
    return MDELAST_OK;
}

void mdelast_mlp_destroy(mdelast_mlp *m) { delete m; }

int mdelast_mlp_n_params(const mdelast_mlp *m, int64_t *n) {
    clear_error();
    if (!m || !n)
        return fail(MDELAST_ERR_ARGUMENT, "bad argument");
    *n = m->np;
    return MDELAST_OK;
}

int mdelast_mlp_get_params(mdelast_mlp *m, float *out) {
    clear_error();
    if (!m || !out)
        return fail(MDELAST_ERR_ARGUMENT, "bad argument");
    MCK(cudaSetDevice(m->device));
    MCK(cudaStreamSynchronize(m->stream));
    MCK(cudaMemcpy(out, m->p, sizeof(float) * static_cast<size_t>(m->np),
                   cudaMemcpyDeviceToHost));
    return MDELAST_OK;
}

int mdelast_mlp_set_params(mdelast_mlp *m, const float *in) {
    clear_error();
    if (!m || !in)
        return fail(MDELAST_ERR_ARGUMENT, "bad argument");
    MCK(cudaSetDevice(m->device));
    MCK(cudaStreamSynchronize(m->stream));
    size_t const bytes = sizeof(float) * static_cast<size_t>(m->np);
    MCK(cudaMemcpy(m->p, in, bytes, cudaMemcpyHostToDevice));
    MCK(cudaMemset(m->m1, 0, bytes)); // a new starting point resets the optimiser
    MCK(cudaMemset(m->m2, 0, bytes));
    MCK(cudaMemset(m->t, 0, sizeof(int)));
    return MDELAST_OK;
}

int mdelast_mlp_forward(mdelast_mlp *m, const float *x, int32_t n, float *y) {
    clear_error();
    if (!m || !x || !y || n < 1)
        return fail(MDELAST_ERR_ARGUMENT, "bad argument");
    MCK(cudaSetDevice(m->device));
    if (int rc = m->upload(x, nullptr, n))
        return rc;
    m->forward(n, m->stream);
    MCK(cudaGetLastError());
    MCK(cudaMemcpyAsync(y, m->A[m->L], sizeof(float) * static_cast<size_t>(n) * m->w[m->L],
                        cudaMemcpyDeviceToHost, m->stream));
    MCK(cudaStreamSynchronize(m->stream));
    return MDELAST_OK;
}

int mdelast_mlp_gradients(mdelast_mlp *m, const float *x, const float *y, int32_t n,
                          float *loss, float *grad) {
    clear_error();
    if (!m || !x || !y || n < 1)
        return fail(MDELAST_ERR_ARGUMENT, "bad argument");
    MCK(cudaSetDevice(m->device));
    if (int rc = m->upload(x, y, n))
        return rc;
    m->forward(n, m->stream);
    m->backward(n, m->stream);
    MCK(cudaGetLastError());
    if (loss)
        MCK(cudaMemcpyAsync(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    if (grad)
        MCK(cudaMemcpyAsync(grad, m->g, sizeof(float) * static_cast<size_t>(m->np),
                            cudaMemcpyDeviceToHost, m->stream));
    MCK(cudaStreamSynchronize(m->stream));
    return MDELAST_OK;
}

int mdelast_mlp_train(mdelast_mlp *m, const float *x, const float *y, int32_t n,
                      int32_t steps, float lr, float *loss) {
    clear_error();
    if (!m || !x || !y || n < 1 || steps < 0 || !(lr > 0.f))
        return fail(MDELAST_ERR_ARGUMENT, "bad argument");
    MCK(cudaSetDevice(m->device));
    if (int rc = m->upload(x, y, n))
        return rc;
    if (!m->graph || m->graph_n != n || m->graph_lr != lr) {
        if (m->graph) {
            cudaGraphExecDestroy(m->graph);
            m->graph = nullptr;
        }
        cudaGraph_t gr = nullptr;
        MCK(cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal));
        m->forward(n, m->stream);
        m->backward(n, m->stream);
        k_adam<<<blocks(m->np), kT, 0, m->stream>>>(m->p, m->g, m->m1, m->m2,
                                                    static_cast<int>(m->np), lr, m->t);
        k_step_inc<<<1, 32, 0, m->stream>>>(m->t);
        cudaError_t const e = cudaStreamEndCapture(m->stream, &gr);
        if (e != cudaSuccess)
            return fail(MDELAST_ERR_CUDA, "capturing the training step: %s",
                        cudaGetErrorString(e));
        cudaError_t const e2 = cudaGraphInstantiate(&m->graph, gr, 0);
        cudaGraphDestroy(gr);
        if (e2 != cudaSuccess)
            return fail(MDELAST_ERR_CUDA, "instantiating the training step: %s",
                        cudaGetErrorString(e2));
        m->graph_n = n;
        m->graph_lr = lr;
    }
    for (int k = 0; k < steps; ++k)
        MCK(cudaGraphLaunch(m->graph, m->stream));
    if (loss) {
        // the loss of the parameters after the last step
        m->forward(n, m->stream);
        m->backward(n, m->stream);
        MCK(cudaMemcpyAsync(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    }
    MCK(cudaStreamSynchronize(m->stream));
    return MDELAST_OK;
}

} // extern "C"
