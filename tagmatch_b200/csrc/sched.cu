// Training and inference kernels of the learned cost model (sched.cuh).
//
// Forward: one thread per sample, the 4,801 parameters in shared memory
// (every thread reads the same weight at the same time: broadcast), the
// first hidden layer in registers.
//
// Gradient: a CTA takes 128 samples.  Phase 1, one thread per sample: the
// forward pass, keeping the first layer's activations H1, the second
// layer's ReLU outputs R2 and the output error DY in shared memory, and the
// error back-propagated to the first layer (DH1).  Phase 2, the CTA's
// threads together: the weight gradients as sums over the 128 samples
// (dW2 = G2^T H1 in 4 x 8 register blocks, G2 = DY W3 [R2 > 0]), written
// as this CTA's partial.  A second kernel sums the partials in a fixed
// order (deterministic), and an Adam kernel updates the parameters.
// Loss: mean squared error over the mini-batch.
#include "sched.cuh"
#include "match.cuh"
#include <chrono>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>

namespace tmb {
namespace {

constexpr int kFwdThreads = 128;
constexpr int kGradSamples = 128;  // samples (and threads) per gradient CTA
constexpr int kRow = kMlpHidden + 1;  // padded row of the per-sample activation arrays

__global__ void __launch_bounds__(kFwdThreads) k_mlp_forward(const float *__restrict__ params, const float *__restrict__ x,
                                                             uint32_t n, float mu, float sigma, float *__restrict__ y) {
    __shared__ float P[kMlpParams];
    for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) P[i] = params[i];
    __syncthreads();
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    float xi[kMlpIn];
#pragma unroll
    for (int k = 0; k < kMlpIn; ++k) xi[k] = x[size_t(s) * kMlpIn + k];
    float h1[kMlpHidden];
#pragma unroll
    for (int i = 0; i < kMlpHidden; ++i) {
        float a = P[kMlpB1 + i];
#pragma unroll
        for (int k = 0; k < kMlpIn; ++k) a = fmaf(P[kMlpW1 + i * kMlpIn + k], xi[k], a);
        h1[i] = fmaxf(a, 0.f);
    }
    float out = P[kMlpB3];
    for (int j = 0; j < kMlpHidden; ++j) {
        float a = P[kMlpB2 + j];
#pragma unroll
        for (int i = 0; i < kMlpHidden; ++i) a = fmaf(P[kMlpW2 + j * kMlpHidden + i], h1[i], a);
        out = fmaf(P[kMlpW3 + j], fmaxf(a, 0.f), out);
    }
    y[s] = out * sigma + mu;
}

struct GradSmem {
    float P[kMlpParams];
    float X[kGradSamples][kMlpIn + 1];
    float H1[kGradSamples][kRow];
    float R2[kGradSamples][kRow];  // ReLU outputs, then G2 = DY W3 [R2 > 0]
    float DH1[kGradSamples][kRow];
    float DY[kGradSamples];
    float red[kGradSamples / 32];
};

// Gradient of (scale / 2) * sum over the CTA's samples of (y - t)^2, i.e.
// of the mean squared error when scale = 2 / batch.  Samples
// [first, first + 128 * gridDim.x) of x / t, with first = sample0 or, when
// step is given, (*step mod steps_per_epoch) * batch (a graph replays the
// same launch for every mini-batch).  partials: [gridDim.x][kMlpParams + 1],
// the last entry the CTA's sum of squared errors.
__global__ void __launch_bounds__(kGradSamples) k_mlp_grad(const float *__restrict__ params, const float *__restrict__ x,
                                                           const float *__restrict__ t, uint32_t n, uint32_t sample0,
                                                           const int *__restrict__ step, uint32_t steps_per_epoch,
                                                           uint32_t batch, float scale, float *__restrict__ partials) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    GradSmem &S = *reinterpret_cast<GradSmem *>(smem_raw);
    const int tid = threadIdx.x;
    for (int i = tid; i < kMlpParams; i += blockDim.x) S.P[i] = params[i];
    const uint32_t first = step ? uint32_t(*step % int(steps_per_epoch)) * batch : sample0;
    const uint32_t s = first + blockIdx.x * kGradSamples + tid;
    const bool valid = s < n && (step == nullptr || blockIdx.x * kGradSamples + tid < batch);
    float xi[kMlpIn];
#pragma unroll
    for (int k = 0; k < kMlpIn; ++k) {
        xi[k] = valid ? x[size_t(s) * kMlpIn + k] : 0.f;
        S.X[tid][k] = xi[k];
    }
    __syncthreads();
    // phase 1: forward and backward of this thread's sample
    float h1[kMlpHidden];
#pragma unroll
    for (int i = 0; i < kMlpHidden; ++i) {
        float a = S.P[kMlpB1 + i];
#pragma unroll
        for (int k = 0; k < kMlpIn; ++k) a = fmaf(S.P[kMlpW1 + i * kMlpIn + k], xi[k], a);
        h1[i] = fmaxf(a, 0.f);
        S.H1[tid][i] = h1[i];
    }
    float out = S.P[kMlpB3];
    for (int j = 0; j < kMlpHidden; ++j) {
        float a = S.P[kMlpB2 + j];
#pragma unroll
        for (int i = 0; i < kMlpHidden; ++i) a = fmaf(S.P[kMlpW2 + j * kMlpHidden + i], h1[i], a);
        const float r = fmaxf(a, 0.f);
        S.R2[tid][j] = r;
        out = fmaf(S.P[kMlpW3 + j], r, out);
    }
    const float err = valid ? out - t[s] : 0.f;
    const float dy = scale * err;
    S.DY[tid] = dy;
    float dh1[kMlpHidden];
#pragma unroll
    for (int i = 0; i < kMlpHidden; ++i) dh1[i] = 0.f;
    for (int j = 0; j < kMlpHidden; ++j) {
        const float g = S.R2[tid][j] > 0.f ? dy * S.P[kMlpW3 + j] : 0.f;
#pragma unroll
        for (int i = 0; i < kMlpHidden; ++i) dh1[i] = fmaf(g, S.P[kMlpW2 + j * kMlpHidden + i], dh1[i]);
    }
#pragma unroll
    for (int i = 0; i < kMlpHidden; ++i) S.DH1[tid][i] = h1[i] > 0.f ? dh1[i] : 0.f;
    // squared error of the CTA
    float se = err * err;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) se += __shfl_xor_sync(0xFFFFFFFFu, se, o);
    if ((tid & 31) == 0) S.red[tid >> 5] = se;
    __syncthreads();
    float *out_p = partials + size_t(blockIdx.x) * (kMlpParams + 1);
    // phase 2: weight gradients, sums over the CTA's samples
    if (tid < kMlpHidden) {  // dW3[j] = sum DY R2[:, j]
        float acc = 0.f;
        for (int q = 0; q < kGradSamples; ++q) acc = fmaf(S.DY[q], S.R2[q][tid], acc);
        out_p[kMlpW3 + tid] = acc;
    } else if (tid == kMlpHidden) {
        float acc = 0.f, l = 0.f;
        for (int q = 0; q < kGradSamples; ++q) acc += S.DY[q];
        for (int w = 0; w < kGradSamples / 32; ++w) l += S.red[w];
        out_p[kMlpB3] = acc;
        out_p[kMlpParams] = l;
    }
    __syncthreads();
    {  // R2 -> G2 (this thread's sample row)
        const float d = S.DY[tid];
        for (int j = 0; j < kMlpHidden; ++j) S.R2[tid][j] = S.R2[tid][j] > 0.f ? d * S.P[kMlpW3 + j] : 0.f;
    }
    __syncthreads();
    {  // dW2[j][i] = sum G2[:, j] H1[:, i]: thread tid owns j in 4 jb .. 4 jb + 3, i in 8 ib .. 8 ib + 7
        const int jb = tid >> 3, ib = tid & 7;
        float acc[4][8];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 8; ++b) acc[a][b] = 0.f;
        for (int q = 0; q < kGradSamples; ++q) {
            float g[4], h[8];
#pragma unroll
            for (int a = 0; a < 4; ++a) g[a] = S.R2[q][4 * jb + a];
#pragma unroll
            for (int b = 0; b < 8; ++b) h[b] = S.H1[q][8 * ib + b];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 8; ++b) acc[a][b] = fmaf(g[a], h[b], acc[a][b]);
        }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 8; ++b) out_p[kMlpW2 + (4 * jb + a) * kMlpHidden + 8 * ib + b] = acc[a][b];
    }
    if (tid < kMlpHidden) {  // db2[j] = sum G2[:, j]; db1[i] = sum DH1[:, i]
        float a2 = 0.f, a1 = 0.f;
        for (int q = 0; q < kGradSamples; ++q) {
            a2 += S.R2[q][tid];
            a1 += S.DH1[q][tid];
        }
        out_p[kMlpB2 + tid] = a2;
        out_p[kMlpB1 + tid] = a1;
    }
    {  // dW1[i][k] = sum DH1[:, i] X[:, k]: thread owns i = tid / 2, k in 4 (tid & 1) .. + 3
        const int i = tid >> 1, k0 = (tid & 1) * 4;
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
        for (int q = 0; q < kGradSamples; ++q) {
            const float d = S.DH1[q][i];
#pragma unroll
            for (int k = 0; k < 4; ++k) acc[k] = fmaf(d, S.X[q][k0 + k], acc[k]);
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) out_p[kMlpW1 + i * kMlpIn + k0 + k] = acc[k];
    }
}

// grads[p] = sum over CTAs of partials[c][p] (fixed order); grads[kMlpParams]
// the summed squared error.
__global__ void k_mlp_reduce(const float *__restrict__ partials, uint32_t ctas, float *__restrict__ grads) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > uint32_t(kMlpParams)) return;
    float acc = 0.f;
    for (uint32_t c = 0; c < ctas; ++c) acc += partials[size_t(c) * (kMlpParams + 1) + p];
    grads[p] = acc;
}

// Adam (Kingma & Ba, 2015) with bias correction; t = *step + 1.
__global__ void k_mlp_adam(float *__restrict__ params, const float *__restrict__ grads, float *__restrict__ m,
                           float *__restrict__ v, const int *__restrict__ step, float lr, float b1, float b2, float eps) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kMlpParams) return;
    const float tt = float(*step + 1);
    const float g = grads[p];
    const float mi = b1 * m[p] + (1.f - b1) * g;
    const float vi = b2 * v[p] + (1.f - b2) * g * g;
    m[p] = mi;
    v[p] = vi;
    const float mh = mi / (1.f - powf(b1, tt)), vh = vi / (1.f - powf(b2, tt));
    params[p] -= lr * mh / (sqrtf(vh) + eps);
}

__global__ void k_step_inc(int *step) { ++*step; }

inline unsigned blocks_of(size_t n, unsigned t) { return unsigned((n + t - 1) / t); }

void set_grad_smem() {
    TM_CUDA(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sizeof(GradSmem))));
}

}  // namespace

void CostModel::init(uint64_t seed) {
    params_.assign(kMlpParams, 0.f);
    std::mt19937_64 rng(seed);
    std::normal_distribution<float> nd(0.f, 1.f);
    for (int i = 0; i < kMlpHidden * kMlpIn; ++i) params_[kMlpW1 + i] = nd(rng) * std::sqrt(2.f / kMlpIn);
    for (int i = 0; i < kMlpHidden * kMlpHidden; ++i) params_[kMlpW2 + i] = nd(rng) * std::sqrt(2.f / kMlpHidden);
    for (int i = 0; i < kMlpHidden; ++i) params_[kMlpW3 + i] = nd(rng) * std::sqrt(1.f / kMlpHidden);
    trained_ = false;
}

void CostModel::loss_grad(const float *params, const float *x, const float *t, uint32_t n, float *y, float *grad,
                          float *loss, cudaStream_t st) {
    DevBuf<float> dp, dx, dt, dy, part, dg;
    dp.reserve(kMlpParams);
    dx.reserve(size_t(std::max<uint32_t>(n, 1)) * kMlpIn);
    dt.reserve(std::max<uint32_t>(n, 1));
    dy.reserve(std::max<uint32_t>(n, 1));
    const uint32_t ctas = std::max(1u, blocks_of(n, kGradSamples));
    part.reserve(size_t(ctas) * (kMlpParams + 1));
    dg.reserve(kMlpParams + 1);
    TM_CUDA(cudaMemcpyAsync(dp.p, params, kMlpParams * 4, cudaMemcpyHostToDevice, st));
    if (n) {
        TM_CUDA(cudaMemcpyAsync(dx.p, x, size_t(n) * kMlpIn * 4, cudaMemcpyHostToDevice, st));
        TM_CUDA(cudaMemcpyAsync(dt.p, t, size_t(n) * 4, cudaMemcpyHostToDevice, st));
    }
    set_grad_smem();
    k_mlp_grad<<<ctas, kGradSamples, sizeof(GradSmem), st>>>(dp.p, dx.p, dt.p, n, 0, nullptr, 1, n, n ? 2.f / n : 0.f,
                                                             part.p);
    TM_CHECK_LAUNCH();
    k_mlp_reduce<<<blocks_of(kMlpParams + 1, 256), 256, 0, st>>>(part.p, ctas, dg.p);
    TM_CHECK_LAUNCH();
    if (n) {
        k_mlp_forward<<<blocks_of(n, kFwdThreads), kFwdThreads, 0, st>>>(dp.p, dx.p, n, 0.f, 1.f, dy.p);
        TM_CHECK_LAUNCH();
        TM_CUDA(cudaMemcpyAsync(y, dy.p, size_t(n) * 4, cudaMemcpyDeviceToHost, st));
    }
    std::vector<float> g(kMlpParams + 1);
    TM_CUDA(cudaMemcpyAsync(g.data(), dg.p, (kMlpParams + 1) * 4, cudaMemcpyDeviceToHost, st));
    TM_CUDA(cudaStreamSynchronize(st));
    std::memcpy(grad, g.data(), kMlpParams * 4);
    *loss = n ? g[kMlpParams] / float(n) : 0.f;
}

void CostModel::predict(const float *x, size_t n, float *y, cudaStream_t st) {
    if (params_.empty()) init(1);
    if (n == 0) return;
    DevBuf<float> dp, dx, dy;
    dp.reserve(kMlpParams);
    dx.reserve(n * kMlpIn);
    dy.reserve(n);
    TM_CUDA(cudaMemcpyAsync(dp.p, params_.data(), kMlpParams * 4, cudaMemcpyHostToDevice, st));
    TM_CUDA(cudaMemcpyAsync(dx.p, x, n * kMlpIn * 4, cudaMemcpyHostToDevice, st));
    k_mlp_forward<<<blocks_of(n, kFwdThreads), kFwdThreads, 0, st>>>(dp.p, dx.p, uint32_t(n), mu_, sigma_, dy.p);
    TM_CHECK_LAUNCH();
    TM_CUDA(cudaMemcpyAsync(y, dy.p, n * 4, cudaMemcpyDeviceToHost, st));
    TM_CUDA(cudaStreamSynchronize(st));
}

TrainReport CostModel::train(const float *x, const float *t, size_t n, uint32_t epochs, uint32_t batch, float lr,
                             cudaStream_t st) {
    if (n < 32) throw Error(TM_ERR_INVALID, "cost model: at least 32 timing samples are needed");
    const auto t0 = std::chrono::steady_clock::now();
    if (params_.empty()) init(1);
    batch = std::max<uint32_t>(kGradSamples, (batch / kGradSamples) * kGradSamples);
    // fixed shuffle; the last 10% is held out
    std::vector<uint32_t> perm(n);
    std::iota(perm.begin(), perm.end(), 0u);
    std::mt19937_64 rng(12345);
    std::shuffle(perm.begin(), perm.end(), rng);
    const size_t n_val = std::max<size_t>(1, n / 10), n_tr = n - n_val;
    double mean = 0, var = 0;
    for (size_t i = 0; i < n_tr; ++i) mean += t[perm[i]];
    mean /= double(n_tr);
    for (size_t i = 0; i < n_tr; ++i) var += (t[perm[i]] - mean) * (t[perm[i]] - mean);
    var /= double(n_tr);
    mu_ = float(mean);
    sigma_ = float(std::sqrt(std::max(var, 1e-12)));
    std::vector<float> hx(n * kMlpIn), ht(n);
    for (size_t i = 0; i < n; ++i) {
        std::memcpy(&hx[i * kMlpIn], x + size_t(perm[i]) * kMlpIn, kMlpIn * 4);
        ht[i] = float((t[perm[i]] - mean) / sigma_);
    }
    const uint32_t steps_per_epoch = uint32_t(std::max<size_t>(1, n_tr / batch));
    const uint32_t ctas = batch / kGradSamples;
    DevBuf<float> dp, dg, dm, dv, part, dx, dt, dy;
    DevBuf<int> dstep;
    dp.reserve(kMlpParams);
    dg.reserve(kMlpParams + 1);
    dm.reserve(kMlpParams);
    dv.reserve(kMlpParams);
    part.reserve(size_t(ctas) * (kMlpParams + 1));
    dx.reserve(n * kMlpIn);
    dt.reserve(n);
    dy.reserve(n);
    dstep.reserve(1);
    TM_CUDA(cudaMemcpyAsync(dp.p, params_.data(), kMlpParams * 4, cudaMemcpyHostToDevice, st));
    TM_CUDA(cudaMemsetAsync(dm.p, 0, kMlpParams * 4, st));
    TM_CUDA(cudaMemsetAsync(dv.p, 0, kMlpParams * 4, st));
    TM_CUDA(cudaMemsetAsync(dstep.p, 0, sizeof(int), st));
    TM_CUDA(cudaMemcpyAsync(dx.p, hx.data(), n * kMlpIn * 4, cudaMemcpyHostToDevice, st));
    TM_CUDA(cudaMemcpyAsync(dt.p, ht.data(), n * 4, cudaMemcpyHostToDevice, st));
    set_grad_smem();
    // one training step as a CUDA graph: gradient of mini-batch (*step mod
    // steps_per_epoch), reduction, Adam, step + 1
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t cs = nullptr;
    TM_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    TM_CUDA(cudaStreamSynchronize(st));
    try {
        TM_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
        k_mlp_grad<<<ctas, kGradSamples, sizeof(GradSmem), cs>>>(dp.p, dx.p, dt.p, uint32_t(n_tr), 0, dstep.p,
                                                                 steps_per_epoch, batch, 2.f / batch, part.p);
        k_mlp_reduce<<<blocks_of(kMlpParams + 1, 256), 256, 0, cs>>>(part.p, ctas, dg.p);
        k_mlp_adam<<<blocks_of(kMlpParams, 256), 256, 0, cs>>>(dp.p, dg.p, dm.p, dv.p, dstep.p, lr, 0.9f, 0.999f, 1e-8f);
        k_step_inc<<<1, 1, 0, cs>>>(dstep.p);
        TM_CUDA(cudaStreamEndCapture(cs, &graph));
        TM_CUDA(cudaGraphInstantiate(&exec, graph, 0));
        const uint64_t steps = uint64_t(steps_per_epoch) * epochs;
        for (uint64_t i = 0; i < steps; ++i) TM_CUDA(cudaGraphLaunch(exec, cs));
        TM_CUDA(cudaStreamSynchronize(cs));
    } catch (...) {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        cudaStreamDestroy(cs);
        throw;
    }
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    cudaStreamDestroy(cs);
    TM_CUDA(cudaMemcpyAsync(params_.data(), dp.p, kMlpParams * 4, cudaMemcpyDeviceToHost, st));
    // errors on the training and validation parts (standardised targets)
    k_mlp_forward<<<blocks_of(n, kFwdThreads), kFwdThreads, 0, st>>>(dp.p, dx.p, uint32_t(n), 0.f, 1.f, dy.p);
    TM_CHECK_LAUNCH();
    std::vector<float> hy(n);
    TM_CUDA(cudaMemcpyAsync(hy.data(), dy.p, n * 4, cudaMemcpyDeviceToHost, st));
    TM_CUDA(cudaStreamSynchronize(st));
    TrainReport r;
    double se_tr = 0, se_val = 0, vm = 0, vv = 0;
    for (size_t i = 0; i < n_tr; ++i) se_tr += double(hy[i] - ht[i]) * (hy[i] - ht[i]);
    for (size_t i = n_tr; i < n; ++i) vm += ht[i];
    vm /= double(n_val);
    for (size_t i = n_tr; i < n; ++i) {
        se_val += double(hy[i] - ht[i]) * (hy[i] - ht[i]);
        vv += (ht[i] - vm) * (ht[i] - vm);
    }
    r.train_mse = se_tr / double(n_tr);
    r.val_mse = se_val / double(n_val);
    r.mean_mse = vv / double(n_val);
    r.val_r2 = vv > 0 ? 1.0 - se_val / vv : 0.0;
    r.samples = n;
    r.steps = uint64_t(steps_per_epoch) * epochs;
    r.ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    trained_ = true;
    return r;
}

// ---------------------------------------------------------------------------
// Scheduler
// ---------------------------------------------------------------------------
void item_features(float *x, uint32_t part_size, uint32_t mask_bits, uint32_t queued, uint32_t chunk_queries,
                   uint32_t seg_tiles_here, float density, uint32_t part_tiles, uint32_t seg_tiles) {
    x[0] = std::log2(1.f + float(part_size)) / 16.f;
    x[1] = float(mask_bits) / 32.f;
    x[2] = std::log2(1.f + float(queued)) / 18.f;
    x[3] = float(chunk_queries) / float(kItemQueries);
    x[4] = std::log2(1.f + float(seg_tiles_here)) / 13.f;
    x[5] = density * 100.f;
    x[6] = float(part_size) / (float(kTile) * float(std::max<uint32_t>(part_tiles, 1)));
    x[7] = std::log2(float(std::max<uint32_t>(seg_tiles, 1))) / 13.f;
}

namespace {
constexpr size_t kMaxSamples = size_t(4) << 20;
constexpr int kTableSteps = 19;  // b = 1 .. 2^18
// candidate tiles per work item (the autotuner's range)
constexpr int kSegChoices = 9;
constexpr uint32_t kSegChoice[kSegChoices] = {32, 64, 128, 256, 512, 1024, 2048, 4096, 8192};

uint32_t mask_bits(const DevTable &t, uint32_t p) {
    uint32_t c = 0;
    for (int k = 0; k < kWords; ++k) c += __builtin_popcount(t.h_part_mask[size_t(p) * 8 + k]);
    return c;
}
}  // namespace

void Scheduler::set_recording(bool on) {
    std::lock_guard<std::mutex> lk(mtx_);
    recording_ = on;
}

bool Scheduler::recording() const {
    std::lock_guard<std::mutex> lk(mtx_);
    return recording_;
}

uint64_t Scheduler::samples() const {
    std::lock_guard<std::mutex> lk(mtx_);
    return t_.size();
}

bool Scheduler::trained() const {
    std::lock_guard<std::mutex> lk(mtx_);
    return model_.trained();
}

void Scheduler::export_samples(float *x, float *t, uint64_t cap, uint64_t *n) const {
    std::lock_guard<std::mutex> lk(mtx_);
    *n = t_.size();
    const uint64_t m = std::min<uint64_t>(cap, t_.size());
    if (x) std::memcpy(x, x_.data(), m * kMlpIn * sizeof(float));
    if (t) std::memcpy(t, t_.data(), m * sizeof(float));
}

void Scheduler::absorb(const DevTable &t, const MatchScratch &s, uint32_t nq, double batch_ms, uint64_t keys) {
    std::lock_guard<std::mutex> lk(mtx_);
    const uint32_t P = t.n_parts;
    if (P == 0 || nq == 0 || s.h_part_count.size() != P) return;
    if (density_.size() != P) {
        density_.assign(P, -1.f);
        frac_.assign(P, 0.f);
    }
    const bool ordered = s.part_order.size() == P;
    const uint32_t seg = s.seg_tiles;
    const bool have_items = !s.h_item_stats.empty() && s.h_item_stats.size() >= 2 * size_t(s.h_item_off[P]);
    std::vector<float> batch_density(P, 0.f);
    if (have_items) {
        for (uint32_t pos = 0; pos < P; ++pos) {
            const uint32_t p = ordered ? s.part_order[pos] : pos;
            const uint32_t cnt = s.h_part_count[p];
            const uint32_t tiles = t.h_part_tiles[p + 1] - t.h_part_tiles[p];
            const uint32_t i0 = s.h_item_off[pos], i1 = s.h_item_off[pos + 1];
            uint64_t recs = 0;
            for (uint32_t i = i0; i < i1; ++i) recs += s.h_item_stats[2 * size_t(i) + 1];
            batch_density[p] = cnt && tiles ? float(double(recs) / (double(cnt) * tiles)) : 0.f;
            if (i1 == i0) continue;
            const float dens = density_[p] >= 0.f ? density_[p] : batch_density[p];
            const uint32_t nch = (cnt + kItemQueries - 1) / kItemQueries;  // chunk groups
            for (uint32_t i = i0; i < i1 && t_.size() < kMaxSamples; ++i) {
                const unsigned long long cyc = s.h_item_stats[2 * size_t(i)];
                if (cyc == 0) continue;
                const uint32_t local = i - i0, chunk = local % nch, sg = local / nch;
                const uint32_t cq = std::min<uint32_t>(kItemQueries, cnt - chunk * kItemQueries);
                const uint32_t ts = std::min<uint32_t>(seg, tiles - sg * seg);
                float f[kMlpIn];
                item_features(f, t.h_part_size[p], mask_bits(t, p), cnt, cq, ts, dens, tiles, seg);
                x_.insert(x_.end(), f, f + kMlpIn);
                t_.push_back(std::log(float(cyc)));
            }
        }
    }
    for (uint32_t p = 0; p < P; ++p) {
        if (have_items) density_[p] = density_[p] >= 0.f ? 0.5f * density_[p] + 0.5f * batch_density[p] : batch_density[p];
        const float fr = float(s.h_part_count[p]) / float(nq);
        frac_[p] = obs_.empty() ? fr : 0.8f * frac_[p] + 0.2f * fr;
    }
    const double kpq = double(keys) / nq;
    keys_per_query_ = obs_.empty() ? kpq : 0.8 * keys_per_query_ + 0.2 * kpq;
    if (obs_.size() < 4096) obs_.push_back({double(nq), batch_ms, double(keys), double(seg)});
}

TrainReport Scheduler::train(const DevTable &t, uint32_t seg_tiles, int sm_count, double clock_hz, uint32_t epochs,
                             cudaStream_t st) {
    std::lock_guard<std::mutex> lk(mtx_);
    TrainReport r = model_.train(x_.data(), t_.data(), t_.size(), epochs, 8192, 1e-3f, st);
    refresh_locked(t, seg_tiles, sm_count, clock_hz, st);
    return r;
}

// Predicted warp-cycles of every partition's items for batches of 2^k
// queries (routed in the recent fractions), for every candidate number of
// tiles per work item, turned into kernel time over the device's matcher
// CTAs: the larger of the summed item time spread over the CTAs and the
// longest item (one CTA runs an item; its 8 warps' cycles add up).  Then a
// least-squares fit of the measured batch times on (1, predicted kernel
// ms, keys).  Also the work-queue order.
void Scheduler::refresh_locked(const DevTable &t, uint32_t seg, int sm_count, double clock_hz, cudaStream_t st) {
    const uint32_t P = t.n_parts;
    if (P == 0 || frac_.size() != P || !model_.trained()) return;
    // rows: [s][k][p][full item, partial item], then the order rows [p]
    const size_t per_seg = size_t(kTableSteps) * P * 2;
    const size_t rows = size_t(kSegChoices) * per_seg + P;
    std::vector<float> x(rows * kMlpIn), y(rows);
    for (int si = 0; si < kSegChoices; ++si) {
        const uint32_t sg = kSegChoice[si];
        for (int k = 0; k < kTableSteps; ++k) {
            const double b = double(1u << k);
            for (uint32_t p = 0; p < P; ++p) {
                const uint32_t tiles = t.h_part_tiles[p + 1] - t.h_part_tiles[p];
                const uint32_t ns = std::max<uint32_t>(1, (tiles + sg - 1) / sg);
                const uint32_t ts = (tiles + ns - 1) / ns;
                const uint32_t cnt = uint32_t(std::llround(b * frac_[p]));
                const float dens = std::max(density_[p], 0.f);
                const size_t r0 = size_t(si) * per_seg + (size_t(k) * P + p) * 2;
                item_features(&x[r0 * kMlpIn], t.h_part_size[p], mask_bits(t, p), cnt, kItemQueries, ts, dens, tiles,
                              sg);
                item_features(&x[(r0 + 1) * kMlpIn], t.h_part_size[p], mask_bits(t, p), cnt,
                              std::max<uint32_t>(1, cnt % kItemQueries), ts, dens, tiles, sg);
            }
        }
    }
    double ref_b = 0;
    for (const auto &o : obs_) ref_b = std::max(ref_b, o[0]);
    if (ref_b <= 0) ref_b = 65536;
    for (uint32_t p = 0; p < P; ++p) {
        const uint32_t tiles = t.h_part_tiles[p + 1] - t.h_part_tiles[p];
        const uint32_t ns = std::max<uint32_t>(1, (tiles + seg - 1) / seg);
        const uint32_t cnt = uint32_t(std::llround(ref_b * frac_[p]));
        item_features(&x[(size_t(kSegChoices) * per_seg + p) * kMlpIn], t.h_part_size[p], mask_bits(t, p), cnt,
                      std::min<uint32_t>(kItemQueries, std::max<uint32_t>(cnt, 1)), (tiles + ns - 1) / ns,
                      std::max(density_[p], 0.f), tiles, seg);
    }
    model_.predict(x.data(), rows, y.data(), st);
    const double ctas = double(std::max(sm_count, 1)) * 4.0;
    table_ms_.assign(size_t(kSegChoices) * kTableSteps, 0.0);
    for (int si = 0; si < kSegChoices; ++si) {
        const uint32_t sg = kSegChoice[si];
        for (int k = 0; k < kTableSteps; ++k) {
            const uint32_t cnt_scale = 1u << k;
            double cyc = 0, longest = 0;
            for (uint32_t p = 0; p < P; ++p) {
                const uint32_t tiles = t.h_part_tiles[p + 1] - t.h_part_tiles[p];
                const uint32_t ns = std::max<uint32_t>(1, (tiles + sg - 1) / sg);
                const size_t r0 = size_t(si) * per_seg + (size_t(k) * P + p) * 2;
                const uint32_t cnt = uint32_t(std::llround(double(cnt_scale) * frac_[p]));
                const uint32_t nf = cnt / kItemQueries, rm = cnt % kItemQueries;
                const double cf = std::exp(double(y[r0])), cr = rm ? std::exp(double(y[r0 + 1])) : 0.0;
                cyc += double(ns) * (nf * cf + cr);
                if (nf) longest = std::max(longest, cf);
                if (rm) longest = std::max(longest, cr);
            }
            // item cycles are summed over the CTA's 8 warps
            table_ms_[size_t(si) * kTableSteps + k] = std::max(cyc / ctas, longest) / 8.0 / clock_hz * 1e3;
        }
    }
    // batch ms = fit0 + fit1 * kernel ms + fit2 * keys / 1e6: least squares
    // with non-negative coefficients (the best of the 7 subsets of terms
    // whose unconstrained solution is non-negative)
    double A[3][3] = {{0}}, B[3] = {0}, YY = 0;
    for (const auto &o : obs_) {
        const double km = kernel_ms_locked(uint32_t(std::max(o[0], 1.0)), uint32_t(o[3]));
        const double v[3] = {1.0, km, o[2] / 1e6};
        for (int i = 0; i < 3; ++i) {
            for (int j = 0; j < 3; ++j) A[i][j] += v[i] * v[j];
            B[i] += v[i] * o[1];
        }
        YY += o[1] * o[1];
    }
    double best_ssr = 1e300;
    double best[3] = {0, 1, 0};
    for (int mask = 1; mask < 8 && !obs_.empty(); ++mask) {
        int idx[3], m = 0;
        for (int i = 0; i < 3; ++i)
            if (mask >> i & 1) idx[m++] = i;
        double M[3][4];
        for (int i = 0; i < m; ++i) {
            for (int j = 0; j < m; ++j) M[i][j] = A[idx[i]][idx[j]] + (i == j ? 1e-9 : 0.0);
            M[i][3] = B[idx[i]];
        }
        bool ok = true;
        for (int c = 0; c < m && ok; ++c) {
            int piv = c;
            for (int r = c + 1; r < m; ++r)
                if (std::fabs(M[r][c]) > std::fabs(M[piv][c])) piv = r;
            if (std::fabs(M[piv][c]) < 1e-15) {
                ok = false;
                break;
            }
            for (int j = 0; j < 4; ++j) std::swap(M[c][j], M[piv][j]);
            for (int r = 0; r < m; ++r) {
                if (r == c) continue;
                const double f = M[r][c] / M[c][c];
                for (int j = 0; j < 4; ++j) M[r][j] -= f * M[c][j];
            }
        }
        if (!ok) continue;
        double c3[3] = {0, 0, 0};
        for (int i = 0; i < m; ++i) c3[idx[i]] = M[i][3] / M[i][i];
        if (c3[0] < 0 || c3[1] < 0 || c3[2] < 0) continue;
        double ssr = YY;
        for (int i = 0; i < 3; ++i) {
            ssr -= 2 * c3[i] * B[i];
            for (int j = 0; j < 3; ++j) ssr += c3[i] * A[i][j] * c3[j];
        }
        if (ssr < best_ssr) {
            best_ssr = ssr;
            std::copy(c3, c3 + 3, best);
        }
    }
    std::copy(best, best + 3, fit_);
    // work-queue order: most expensive items first
    std::vector<float> cost(P);
    for (uint32_t p = 0; p < P; ++p) cost[p] = y[size_t(kSegChoices) * per_seg + p];
    order_.resize(P);
    std::iota(order_.begin(), order_.end(), 0u);
    std::stable_sort(order_.begin(), order_.end(), [&](uint32_t a, uint32_t b) { return cost[a] > cost[b]; });
}

std::vector<uint32_t> Scheduler::order() const {
    std::lock_guard<std::mutex> lk(mtx_);
    return order_;
}

// Predicted kernel ms of a batch of b queries at seg tiles per item (the
// nearest candidate), interpolated between powers of two of b.
double Scheduler::kernel_ms_locked(uint32_t b, uint32_t seg) const {
    if (table_ms_.empty() || b == 0) return 0.0;
    int si = 0;
    for (int i = 1; i < kSegChoices; ++i)
        if (std::fabs(std::log2(double(kSegChoice[i]) / seg)) < std::fabs(std::log2(double(kSegChoice[si]) / seg))) si = i;
    const double *tm = &table_ms_[size_t(si) * kTableSteps];
    const double kb = std::log2(double(b));
    const int k0 = std::min(kTableSteps - 2, int(kb));
    const double fr = std::min(1.0, kb - k0);
    return tm[k0] * std::pow(tm[k0 + 1] / std::max(tm[k0], 1e-9), fr);
}

uint32_t Scheduler::best_seg_locked(uint32_t b) const {
    uint32_t best = kSegChoice[0];
    double best_ms = 1e300;
    for (int i = 0; i < kSegChoices; ++i) {
        const double ms = kernel_ms_locked(b, kSegChoice[i]);
        if (ms < best_ms) {
            best_ms = ms;
            best = kSegChoice[i];
        }
    }
    return best;
}

uint32_t Scheduler::best_seg(uint32_t b) const {
    std::lock_guard<std::mutex> lk(mtx_);
    return table_ms_.empty() ? 0u : best_seg_locked(b);
}

double Scheduler::model_batch_ms_locked(uint32_t b) const {
    const double km = kernel_ms_locked(b, best_seg_locked(b));
    return fit_[0] + fit_[1] * km + fit_[2] * keys_per_query_ * b / 1e6;
}

double Scheduler::predict_batch_ms(uint32_t b) const {
    std::lock_guard<std::mutex> lk(mtx_);
    if (table_ms_.empty() || b == 0) return 0.0;
    const int k = std::min(kTableSteps - 1, int(std::log2(double(b))));
    return model_batch_ms_locked(b) * correction_[k];
}

void Scheduler::observe_batch(uint32_t b, double ms) {
    std::lock_guard<std::mutex> lk(mtx_);
    if (table_ms_.empty() || b == 0 || ms <= 0) return;
    const double pred = model_batch_ms_locked(b);
    if (pred <= 0) return;
    const int k = std::min(kTableSteps - 1, int(std::log2(double(b))));
    correction_[k] = 0.9 * correction_[k] + 0.1 * std::min(8.0, std::max(0.125, ms / pred));
}

uint32_t Scheduler::stable_batch(double rate_qps, uint32_t cap, int lanes) const {
    if (cap <= 1 || rate_qps <= 0) return 1;
    // steps of 2^(1/4); the lanes' batches run side by side, and the batch
    // times were measured that way
    for (double b = 1; b < cap; b *= 1.189207115) {
        const uint32_t bi = uint32_t(b);
        const double ms = predict_batch_ms(bi);
        if (ms > 0 && lanes * bi / ms * 1e3 >= 1.25 * rate_qps) return bi;
    }
    return cap;
}

}  // namespace tmb
