// warm.h -- reduced-basis learned warm start (warm.cu).
#pragma once

#include "common.h"
#include "mlp.h"

namespace fg
{

class WarmModel
{
public:
  // mean [N], basis [rank][N] (orthonormal rows), the network (borrowed; its outputs = rank)
  // and the input / output normalisation.  mlp may be null for projection only.
  Status Create(int N, int rank, const double *mean, const double *basis, Mlp *mlp,
                const float *feature_shift, const float *feature_scale, const double *coeff_shift,
                const double *coeff_scale);
  int N() const { return N_; }
  int rank() const { return rank_; }
  int inputs() const { return mlp_ ? mlp_->inputs() : 0; }
  int64_t launches() const { return launches_; }

  Status Project(int k, const double *a_host, double *coeffs_host);
  Status ProjectDevice(int k, const double *a, double *coeffs, cudaStream_t stream);
  Status Predict(int k, const float *features_host, double *a_host);
  Status PredictDevice(int k, const float *features, double *a, cudaStream_t stream);

private:
  int N_ = 0, rank_ = 0;
  int64_t launches_ = 0;
  Mlp *mlp_ = nullptr;
  DeviceArray<double> mean_, basis_, cshift_, cscale_, a_;
  DeviceArray<float> fshift_, fscale_, xn_, y_, f_;
};

} // namespace fg

struct fg_warm {
  fg::WarmModel warm;
  fg::DeviceArray<float> features; // staging for fg_solve_batch_learned
  fg::DeviceArray<double> starts;
};
