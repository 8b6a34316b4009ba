// Learned control variate for the exchange energy (internal interface).
#pragma once
#include <functional>
#include "afq_common.cuh"

namespace afq {

struct Mlp;
cudaError_t mlp_create(int nin, int H, int cap, unsigned long long seed, Mlp** out,
                       cudaStream_t st);
void mlp_destroy(Mlp* m);
long long mlp_nparams(const Mlp* m);
int mlp_capacity(const Mlp* m);
float* mlp_x(Mlp* m);
float* mlp_t(Mlp* m);
float* mlp_y(Mlp* m);
cudaError_t mlp_set_params(Mlp* m, const float* host, cudaStream_t st);
cudaError_t mlp_get_params(Mlp* m, float* host, cudaStream_t st);
cudaError_t mlp_forward(Mlp* m, const float* x, int B, float* y, bool keep, cudaStream_t st);
cudaError_t mlp_gradient(Mlp* m, const float* x, const float* t, int B, cudaStream_t st);
// last_loss: host destination of the last step's loss (pinned when !sync_loss, then the
// copy is left in flight on st).
cudaError_t mlp_train(Mlp* m, const float* x, const float* t, int B, int iters, float lr,
                      float* last_loss, cudaStream_t st, bool sync_loss = true);
// Rescales the network so that it computes the same function of new input / output
// coordinates: x_old = a * x_new + c (device arrays [nin]), y_new = alpha y_old + gamma.
// Restarts the Adam moments.
cudaError_t mlp_restandardize(Mlp* m, const float* a, const float* c, float alpha, float gamma,
                              cudaStream_t st);

struct CvConfig {
  int hidden = 256;
  float lr = 1e-3f;
  unsigned long long seed = 12345;
  long long train_walker_steps = 2000;   // exact samples gathered before the estimator
  int subset_den = 8;                     // exact exchange on nw / subset_den walkers
  int iters_warm = 200, iters_online = 20;
  int batch_online = 1024;                // samples per online Adam step (a window of the buffer)
  // subset design: 0 = simple random sample of m walkers (inclusion m / nw); 1 = systematic
  // sample of m teeth with probability proportional to the walker weight, over the walkers
  // ordered by the surrogate's prediction (implicit stratification)
  int sampling = 1;
  // linearised exchange: Q = dE_K/dG at the weighted-mean G of the first measurement, and
  // again every q_refresh measurements (0: never again); features 36/37 are the linearised
  // E_K(G_w) = E_K(Gm) + Q.(G_w - Gm) (Re relative to the first one, Im)
  int q_refresh = 0;
  // residual learning: the network predicts E_K minus feature 36 (the linearisation)
  int residual = 0;
  // low-precision base: the exchange of every walker from one plain bf16 tensor-core
  // product (CvInputs::base_exchange) takes the place of the linearisation in features
  // 36/37 and the network learns E_K minus it (residual learning on)
  int base = 0;
};

struct CvState;

// Device inputs of one measurement.  exact_exchange(Gc_sub, m, Kpart) must write the
// exchange partial sums [m][2][nblk] of the m walkers whose compact density matrices
// are packed in Gc_sub.
struct CvInputs {
  const z_t* Gc;        // [nw][NAK]
  const z_t* haj;       // [NAK]
  const z_t* cvec;      // [nchol][nw], Coulomb vector of every walker
  z_t* Wd;              // [nw][8] walker data (overlaps in 2, 3; eloc written to 0)
  z_t* Kpart;           // [nw][2][nblk] scratch for the exact exchange
  int nblk;
  std::function<cudaError_t(const z_t*, int, z_t*)> exact_exchange;
  const z_t* Lh;        // [nchol][2][n][N] unscaled half-rotated factors (FP64)
  int n, N;
  // base_exchange(Gc, nw, Kpart): low-precision exchange partial sums of every walker, in
  // the layout of exact_exchange (empty: no low-precision base available)
  std::function<cudaError_t(const z_t*, int, z_t*)> base_exchange;
};

cudaError_t cv_create(const CvConfig& cfg, int nw, int nchol, long long nak, CvState** out,
                      cudaStream_t st);
void cv_destroy(CvState* s);
// Runs one measurement; writes W_data[:,0] and the two weighted sums (sum Re(e) Re(w),
// sum Re(w)) of the estimator.  Synchronises the stream; the network's online training
// steps are left running on the estimator's own stream (cv_sync waits for them).
cudaError_t cv_energy(CvState* s, const CvInputs& in, double* sums, cudaStream_t st);
// stats: [exact samples seen, subset size of the last measurement, last training loss,
//         estimator active (0/1), measurements, sampling variance of the last estimate
//         from the subset correction, re-standardisations, fallback to exact (0/1)]
void cv_stats(CvState* s, double* stats);
// Waits for the online training left running after the last measurement.
cudaError_t cv_sync(CvState* s);
// Kernels launched by the last cv_energy call (training included).
long long cv_launches(const CvState* s);
// Surrogate exchange energy of every walker from the last measurement (host doubles).
cudaError_t cv_predictions(CvState* s, double* host, cudaStream_t st);

}  // namespace afq
