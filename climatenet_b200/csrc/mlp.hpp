// mlp.hpp — the per-contact warm-start network (mlp.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "device.cuh"

namespace pdfb {

constexpr int kMlpIn = 10, kMlpHidden = 64, kMlpOut = 3;
constexpr int kMlpParams = kMlpHidden * kMlpIn + kMlpHidden + kMlpHidden * kMlpHidden + kMlpHidden +
                           kMlpOut * kMlpHidden + kMlpOut;  // 5,059

// Device entry points (all on stream st; buffers are device pointers).
void mlp_forward_device(const float* prm, const float* X, int n, float* Y, cudaStream_t st);
// Same, for min(*n_dev, cap) samples whose count lives on the device.
void mlp_forward_counted(const float* prm, const float* X, const int* n_dev, int cap, float* Y, cudaStream_t st);
// Accumulates d(mean squared error)/d(params) of samples idx[0..n) (0..n when
// idx is null) into grad and the loss into *loss (both must be zeroed first).
void mlp_grad_device(const float* prm, const float* X, const float* T, const int* idx, int n, float* grad,
                     double* loss, cudaStream_t st);
// Adam on device: step is the 1-based update count.
void mlp_adam_device(float* prm, const float* grad, float* m1, float* m2, double lr, int64_t step, cudaStream_t st);

// Trains prm (device, in place) on the n samples X (n x 10), T (n x 3), both
// device-resident: seeded shuffle, 90/10 split, `epochs` passes of Adam over
// the training part in mini-batches.  Returns the mean training loss of the
// last epoch; *val_loss gets the loss on the held-out part.
double mlp_train_device(float* prm, const float* X, const float* T, int n, int epochs, int batch, double lr,
                        uint64_t seed, double* val_loss, cudaStream_t st);

// Seeded He initialisation of a parameter vector (host; defined in api.cu).
void mlp_init_params(float* w, uint64_t seed);
// Same as mlp_train_device on standardised copies of the samples (per-column
// mean and standard deviation, the constant bias feature left alone),
// starting from a seeded He initialisation; the standardisation is folded
// back into the first and last layers of prm, so the network takes raw
// features and returns raw forces.  Losses are those of the standardised
// problem (1.0 = predicting the mean).
double mlp_train_standardized(float* prm, const float* X, const float* T, int n, int epochs, int batch, double lr,
                              uint64_t seed, double* val_loss, cudaStream_t st);

// Warm-start kernels of the step loop.
//  features of every obstacle contact (requires c.c_gap, t_n and the r_prev memory)
void launch_mlp_features(cudaStream_t st, DContacts c, const double* tn, const double* mass, const double* rprev,
                         const int* rprev_tag, int tag_prev, const double g[3], double dt, float* X);
//  end of step: r_prev memory of the contact vertices, optional sample log
void launch_mlp_record(cudaStream_t st, DContacts c, const double* mass, double* rprev, int* rprev_tag, int tag,
                       const double g[3], double dt, const float* X, float* SX, float* ST, int* n_samples, int cap);

}  // namespace pdfb
