// mlp.h -- dense MLP (inputs -> hidden -> hidden -> outputs, GELU hidden layers) trained
// and evaluated on the GPU by this library's kernels (mlp.cu), in FP32.
#pragma once

#include "common.h"

#include <cstdint>

namespace fg
{

class Mlp
{
public:
  Status Create(int inputs, int hidden, int outputs, uint64_t seed);
  int64_t ParameterCount() const;
  int inputs() const { return I_; }
  int hidden() const { return H_; }
  int outputs() const { return O_; }
  int64_t launches() const { return launches_; }

  Status GetParameters(float *host) const;
  Status SetParameters(const float *host);
  // y = f(x), host arrays [batch][inputs] -> [batch][outputs].
  Status Predict(int batch, const float *x_host, float *y_host);
  // y = f(x), device arrays, on `stream`.
  Status PredictDevice(int batch, const float *x_dev, float *y_dev, cudaStream_t stream);
  // Loss 0.5 / batch * sum (f(x) - t)^2 and its gradient (parameter layout).
  Status LossGradient(int batch, const float *x_host, const float *t_host, float *loss,
                      float *gradient_host);
  // Adam on shuffled minibatches of a device copy of (x, t); final_loss over all samples.
  Status Train(int samples, const float *x_host, const float *t_host, int epochs, int batch,
               float learning_rate, uint64_t seed, float *final_loss);

private:
  struct Views {
    float *w1, *b1, *w2, *b2, *w3, *b3;
  };
  Views Split(float *q) const;
  Status EnsureBatch(int batch);
  Status Forward(int batch, const float *x, float *y, cudaStream_t st);
  Status Backward(int batch, const float *x, const float *t, cudaStream_t st);

  int I_ = 0, H_ = 0, O_ = 0;
  int batch_cap_ = 0;
  int64_t steps_ = 0, launches_ = 0;
  DeviceArray<float> p_, g_, m_, v_;
  DeviceArray<float> x_, t_, h1_, a1_, h2_, a2_, y_, dy_, d2_, d1_, row_loss_, loss_;
};

} // namespace fg

struct fg_mlp {
  fg::Mlp mlp;
};
