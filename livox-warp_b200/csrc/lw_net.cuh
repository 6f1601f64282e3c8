// Internal interface between the learned-start-pose network (lw_initnet.cu) and the odometry (lw_odom.cu).
#pragma once
#include "lw_common.cuh"

namespace lw {

// The two point sets of a frame in the frame of the device pose T (lw_net_sets without the argument checks).
int net_sets_launch(const float* ds_xyz, const int32_t* n_ds, const lw_regmap& reg, const double* T, float radius,
                    float voxel, float* sets, int32_t* cand, int32_t* tiles, int32_t* count, cudaStream_t s);

// Forward pass of n samples (lw_net_forward without the argument checks).
int net_forward_launch(const lw_initnet& net, const float* sets, int n, float* pooled, int32_t* argmax, float* hid,
                       float* step, int32_t* err, cudaStream_t s);

// T_pred = T_reg = T_pred * [R(step_r), step_t] when the frame registers and the forward pass ran cleanly.
int net_apply_launch(lw_odom_state* st, const float* step, const int32_t* err, cudaStream_t s);

}  // namespace lw
