// costmodel.hpp — learned cost model of device operations (costmodel.cu) and its features.
#pragma once

#include <array>
#include <cstdint>
#include <vector>

#include "gates.hpp"

namespace lqcs_b200 {

// Features of one device operation: op kind, width, lowest and highest qubit it touches,
// number of source gates, register size, FP64 flops per amplitude (for a tile pass the
// flops of all its operations: what its time grows with beyond the one HBM round trip).
// Scaled to O(1) by op_features.
constexpr int kCostFeatures = 7;
constexpr int kCostHidden = 64;
constexpr int kCostParams = kCostHidden * kCostFeatures + kCostHidden +
                            kCostHidden * kCostHidden + kCostHidden + kCostHidden + 1;

std::array<float, kCostFeatures> op_features(uint32_t kind, uint32_t width, uint32_t min_target,
                                             uint32_t max_target, uint32_t gates, uint32_t n,
                                             double flops_per_amp);
std::array<float, kCostFeatures> op_features(const DevOp& op, uint32_t n);

// Train from scratch on (features, targets); returns the final mean squared error.
float costmodel_train(const float* features, const float* targets, uint64_t n, uint32_t epochs,
                      float lr, uint64_t seed);
void costmodel_predict(const float* features, uint64_t n, float* out);
// Loss and flattened gradient of the current weights on a batch (no update).
float costmodel_grad(const float* features, const float* targets, uint64_t n, float* grad_out);
std::vector<float> costmodel_weights();
void costmodel_set_weights(const float* w, uint64_t n);
bool costmodel_trained();
void costmodel_clear();
uint64_t costmodel_version();   // changes whenever the weights change

// Predicted device time (ms) of a list of device operations on n qubits.
double predict_ops_ms(const std::vector<DevOp>& ops, uint32_t n);

}  // namespace lqcs_b200
