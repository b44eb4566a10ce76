// Learned SA source: weights, normalisation and training hull on the device.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

namespace phx {

constexpr int kMlpIn = 6;       // input features
constexpr int kMlpK1 = 16;      // first-layer K padded to one MMA
constexpr int kMlpH = 64;       // hidden width
constexpr int kMlpTile = 128;   // cells per CTA tile (MMA M)
constexpr int kMlpGrid = 256;   // occupancy bins per axis over (f0, f1) = (ln chi, ln s) of the training hull

// Occupancy bin of a feature value over [lo, hi] (host and device alike).
__host__ __device__ inline int mlp_bin(float v, float lo, float hi)
{
    if (!(hi > lo)) return 0;
    const float t = (v - lo) / (hi - lo) * (float)kMlpGrid;
    if (!(t >= 0.0f)) return 0;
    return t >= (float)(kMlpGrid - 1) ? kMlpGrid - 1 : (int)t;
}

// Weights as FP16 words in the canonical K-major core-matrix layout the MMA
// reads (byte offset of (n, k) = (n / 8) * sbo + (k / 8) * 128 + (n % 8) * 16 +
// (k % 8) * 2, sbo = 256 for W1 (K = 16), 1024 for W2 and W3 (K = 64)), so a
// CTA copies them to shared memory as they are.
struct MlpDev {
    const uint16_t *w1c;        // [64 x 16]
    const uint16_t *w2c;        // [64 x 64]
    const uint16_t *w3c;        // [64 x 64]
    const float *b1, *b2, *b3;  // [64]
    const float *w4;            // [64]
    float b4;
    float mean[kMlpIn], rstd[kMlpIn];  // feature standardisation
    float lo[kMlpIn], hi[kMlpIn];      // training hull (raw features): the box
    const uint8_t *occ;                // and the occupied (f0, f1) bins [kMlpGrid][kMlpGrid]
    float tscale;                      // target scale
};

// Plain FP32 weights of the trainer, row-major [out][in].
struct MlpHostWeights {
    float w1[kMlpH * kMlpIn], b1[kMlpH];
    float w2[kMlpH * kMlpH], b2[kMlpH];
    float w3[kMlpH * kMlpH], b3[kMlpH];
    float w4[kMlpH], b4;
};

}  // namespace phx
