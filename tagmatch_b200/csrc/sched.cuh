// Learned cost model of the subset test: an 8 -> 64 -> 64 -> 1 fp32 MLP
// (ReLU) that predicts the log of a work item's warp-cycles from features
// of the item and its partition.  Trained on the GPU by the kernels in
// sched.cu (forward, backward, Adam), on timing samples the matcher records
// (k_match's per-item warp-cycles).  The engine uses the predictions to
// order partitions in the persistent kernel's work queue and to set the
// flush points of the learned serving mode; without a trained model the
// autotuner's static choices stand.  The reference has no counterpart: its
// queues flush when full or older than the latency limit
// (front_end.cc:325-376, 563-598).
#pragma once
#include <array>
#include <cstdint>
#include <mutex>
#include <vector>
#include "tm_host.hpp"

namespace tmb {

constexpr int kMlpIn = 8;
constexpr int kMlpHidden = 64;
// parameter layout (floats): W1 [64][8], b1 [64], W2 [64][64] (W2[j][i]:
// output j, input i), b2 [64], W3 [64], b3
constexpr int kMlpW1 = 0;
constexpr int kMlpB1 = kMlpW1 + kMlpHidden * kMlpIn;
constexpr int kMlpW2 = kMlpB1 + kMlpHidden;
constexpr int kMlpB2 = kMlpW2 + kMlpHidden * kMlpHidden;
constexpr int kMlpW3 = kMlpB2 + kMlpHidden;
constexpr int kMlpB3 = kMlpW3 + kMlpHidden;
constexpr int kMlpParams = kMlpB3 + 1;  // 4801

struct TrainReport {
    double train_mse = 0, val_mse = 0, val_r2 = 0, mean_mse = 0;  // on standardised log-cycles
    uint64_t samples = 0, steps = 0;
    double ms = 0;
};

class CostModel {
public:
    // He-initialised weights from a fixed seed.
    void init(uint64_t seed);
    // Trains on n samples (x [n][8], t [n] log-cycles) with mini-batch Adam:
    // 90% train, 10% validation (a fixed shuffle); the whole step (gradient
    // of a mini-batch, its reduction, the Adam update) is one CUDA graph
    // replayed for every mini-batch.
    TrainReport train(const float *x, const float *t, size_t n, uint32_t epochs, uint32_t batch, float lr, cudaStream_t st);
    // Predicted log-cycles (unstandardised) for n feature rows, on the GPU.
    void predict(const float *x, size_t n, float *y, cudaStream_t st);
    bool trained() const { return trained_; }
    const std::vector<float> &params() const { return params_; }

    // For the gradient check: the network's outputs y [n], the gradient of
    // the mean squared error over the n samples w.r.t. every parameter
    // (grad [kMlpParams]) and the loss, computed by the training kernels.
    static void loss_grad(const float *params, const float *x, const float *t, uint32_t n, float *y, float *grad,
                          float *loss, cudaStream_t st);

private:
    std::vector<float> params_;
    float mu_ = 0, sigma_ = 1;  // target standardisation
    bool trained_ = false;
};

struct DevTable;
struct MatchScratch;

// Features of one work item (inputs of the cost model), each scaled to
// about [0, 1]: partition size, partition mask popcount (the length of the
// partition's common prefix in the reference's terms), queries queued for
// the partition, queries in the item's chunk, tiles in the item's segment,
// recent match density of the partition (hit records per (query, tile)),
// filters per tile of the partition, tiles per work item.
void item_features(float *x, uint32_t part_size, uint32_t mask_bits, uint32_t queued, uint32_t chunk_queries,
                   uint32_t seg_tiles_here, float density, uint32_t part_tiles, uint32_t seg_tiles);

// The learned scheduler: timing samples, the cost model, and the decisions
// taken from it (work-queue order, predicted batch time for flush points).
class Scheduler {
public:
    void set_recording(bool on);
    bool recording() const;
    // One matched batch: its per-item timings (s.h_item_stats, in queue
    // order) become samples; per-partition routing fractions and match
    // densities are updated; (queries, host-measured ms, keys) is kept for
    // the batch-time fit.
    void absorb(const DevTable &t, const MatchScratch &s, uint32_t nq, double batch_ms, uint64_t keys);
    uint64_t samples() const;
    void export_samples(float *x, float *t, uint64_t cap, uint64_t *n) const;
    // Trains the cost model on every sample so far, then refreshes the
    // decisions for table t.
    TrainReport train(const DevTable &t, uint32_t seg_tiles, int sm_count, double clock_hz, uint32_t epochs,
                      cudaStream_t st);
    bool trained() const;
    // Partitions in descending order of predicted item cost.
    std::vector<uint32_t> order() const;
    // Predicted milliseconds of a batch of b queries at its best tiles per
    // work item (0 when untrained).
    double predict_batch_ms(uint32_t b) const;
    // Tiles per work item with the lowest predicted kernel time for a batch
    // of b queries (0 when untrained).
    uint32_t best_seg(uint32_t b) const;
    // A matched batch's measured milliseconds: corrects the predictions
    // online, one factor per power-of-two batch size (moving average of
    // measured over predicted).
    void observe_batch(uint32_t b, double ms);
    // Smallest batch (at most cap) whose predicted throughput -- lanes x
    // queries over predicted batch time, the lanes' batches running side by
    // side -- is at least 1.25 x the arrival rate: batches of that size keep
    // up with the arrivals.
    uint32_t stable_batch(double rate_qps, uint32_t cap, int lanes) const;

private:
    void refresh_locked(const DevTable &t, uint32_t seg_tiles, int sm_count, double clock_hz, cudaStream_t st);
    double kernel_ms_locked(uint32_t b, uint32_t seg) const;
    uint32_t best_seg_locked(uint32_t b) const;
    double model_batch_ms_locked(uint32_t b) const;
    std::array<double, 19> correction_ = [] {
        std::array<double, 19> c{};
        c.fill(1.0);
        return c;
    }();
    mutable std::mutex mtx_;
    bool recording_ = false;
    std::vector<float> x_, t_;                 // samples: features [n][8], log warp-cycles [n]
    std::vector<float> density_, frac_;        // per partition: match density, routed queries per query
    std::vector<std::array<double, 4>> obs_;   // batches: queries, measured ms, keys, tiles per item
    double keys_per_query_ = 0;
    CostModel model_;
    std::vector<uint32_t> order_;
    std::vector<double> table_ms_;             // predicted kernel ms, [tiles-per-item choice][b = 2^k]
    double fit_[3] = {0, 1, 0};                // batch ms = fit0 + fit1 * kernel ms + fit2 * keys / 1e6
};

}  // namespace tmb
