// Learned leaving-row scorer (MLP 12 -> 64 -> 64 -> 1), engine-side declarations.
#pragma once
namespace ds {
struct MlpModel;
// Device pointers the iteration kernels read (bf16 W1, bf16 W2, fp32 parameters, error flag).
void model_pointers(const MlpModel* md, const void** w1, const void** w2, const float** p, int** err);
int model_device(const MlpModel* md);
}  // namespace ds

struct ds_model;
// The model behind a C-ABI handle.
ds::MlpModel* ds_model_impl(ds_model* m);
