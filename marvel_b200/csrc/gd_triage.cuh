// gd_triage.cuh -- learned triage of pair groups: features, and a 12-64-64-1 MLP trained and
// evaluated with BF16 tensor-core kernels (FP32 accumulate, FP32 Adam state).
#pragma once
#include "gd_common.cuh"
#include "gd_filter.cuh"

namespace gd
{

constexpr int TRI_NF = 12;   // features per pair group
constexpr int TRI_H = 64;    // hidden width
// parameter vector (float32): feature mean[12], std[12], W1[64][12], b1[64], W2[64][64], b2[64], W3[64], b3
constexpr int TRI_OFF_MEAN = 0;
constexpr int TRI_OFF_STD = 12;
constexpr int TRI_OFF_W1 = 24;
constexpr int TRI_OFF_B1 = TRI_OFF_W1 + TRI_H * TRI_NF;
constexpr int TRI_OFF_W2 = TRI_OFF_B1 + TRI_H;
constexpr int TRI_OFF_B2 = TRI_OFF_W2 + TRI_H * TRI_H;
constexpr int TRI_OFF_W3 = TRI_OFF_B2 + TRI_H;
constexpr int TRI_OFF_B3 = TRI_OFF_W3 + TRI_H;
constexpr int TRI_NPARAM = TRI_OFF_B3 + 1;  // 5081, of which 5057 trained

// The learned triage of the ng pair groups selection kept (groups[0, ng), each a hit range):
// per group its features (into feat, when given, at the group's slot) and with params !=
// nullptr the MLP's verdict skip[g] = p < threshold (nskip += #skipped).
int launch_triage_groups(const uint2* groups, unsigned ng, const uint64_t* hkey, const uint32_t* hdiag, HitBits hb,
                         const DevBlock& A, const DevBlock& B, int comp, int minover, int binshift,
                         const int64_t* amask_anno, const int32_t* amask_data, const float* params, float threshold,
                         float* feat, uint8_t* skip, unsigned* nskip, cudaStream_t s);

// p[i] = sigmoid(MLP(x[i])) for n rows of TRI_NF features.
int launch_mlp_forward(const float* params, const float* x, int64_t n, float* p, cudaStream_t s);

// Gradient of the weighted binary cross-entropy over one batch (rows x[0..n)); grad has
// TRI_NPARAM floats (zeroed here), loss receives the mean loss.
int launch_mlp_grad(const float* params, const float* x, const float* y, int n, float pos_weight, float* grad,
                    float* loss, cudaStream_t s);

int launch_mlp_grad_perm(const float* params, const float* x, const float* y, const int* perm, int64_t n0, int n,
                         float pos_weight, float* grad, float* loss, cudaStream_t s);

int launch_adam(float* params, const float* grad, float* m, float* v, int step, float lr, cudaStream_t s);

}  // namespace gd
