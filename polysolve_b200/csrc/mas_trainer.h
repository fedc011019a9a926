// Host side of the warm-start network's GPU training (the mas_ws_trainer handle of the C ABI).
//
// The trainer keeps its samples resident in device memory: one banked pattern per sequence of
// systems (shared by the sequence's samples) and, per sample, the FP32 block values, the neighbour
// weights and their mirrored copies, the normalised features, r_g and {s_q, e . r_g}. Samples are
// added from a factorized solver (mas_ws_trainer_add_sample, which runs the solver's own prediction
// pipeline up to the features); training steps, evaluation and gradients run the kernels of
// mas_ws_train.cu on the trainer's stream.
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "mas_internal.h"

struct mas_ws_trainer
{
    struct Pattern
    {
        const void *owner = nullptr; // the solver the pattern came from
        uint64_t key = 0;            // its pattern / ordering identity
        int banks = 0;
        long long slots = 0;
        pmas::DevBuf<long long> slice;
        pmas::DevBuf<int> rowlen, cols, diag_slot, mirror;
        pmas::DevBuf<uint8_t> real;
    };
    struct Sample
    {
        int pattern = 0;
        pmas::DevBuf<float> vals32, wslot, wT, feat;
        pmas::DevBuf<double> re, sc;
    };

    int device = 0;
    cudaStream_t stream = nullptr;
    std::string last_error;
    std::vector<std::unique_ptr<Pattern>> patterns;
    std::vector<std::unique_ptr<Sample>> samples;
    pmas::DevBuf<float> prm, adam_m, adam_v, grad;
    pmas::DevBuf<uint16_t> wl;
    long long steps = 0;

    // Scratch sized for the largest sample.
    int cap_nodes = 0;
    pmas::DevBuf<float> z0, z[pmas::WS_LAYERS], gh, g1, gm, partials;
    pmas::DevBuf<uint16_t> h[pmas::WS_LAYERS + 1], m[pmas::WS_LAYERS];
    pmas::DevBuf<double> c, Ac, red, losses;
    pmas::DevBuf<pmas::WsTrainState> st;
    pmas::DevBuf<double> coll_partials;
    pmas::DevBuf<unsigned> coll_counter;

    ~mas_ws_trainer();
    void init(const float *params, long long count);
    // Index of the stored pattern matching the solver's current one (stored now if new).
    int pattern_for(const void *owner, uint64_t key, const pmas::BankedMatrix &A, const int *diag_slot,
                    cudaStream_t s);
    void add_sample(int pattern, const pmas::BankedMatrix &A, const float *wslot, const float *feat_raw,
                    const pmas::WsState *ws, const double *rg, const pmas::WsHistory &hist, const double *x_exact,
                    size_t len, cudaStream_t s);
    pmas::WsTrainView view(int i) const;
    pmas::WsTrainScratch scratch();
    void ensure_scratch(int nodes);
    void gradient(int i, float *out, double *loss);
    void train(const int *idx, const float *lr, int count, double *loss_out);
    void evaluate(const int *idx, int count, double *rho_out);
};
