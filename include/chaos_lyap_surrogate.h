/* chaos_lyap surrogate: an ensemble of small MLPs (parameter point ->
 * Lyapunov spectrum) trained and evaluated on the GPU by this library's own
 * BF16 tensor-core kernels (FP32 accumulate, FP32 master weights, Adam).  Used
 * to fill smooth regions of fine maps; cells where the ensemble disagrees or
 * the leading exponent is near zero are sent to the sweep (chaos_lyap.h).
 * No counterpart in the reference (it integrates every cell). */
#ifndef CHAOS_LYAP_SURROGATE_H
#define CHAOS_LYAP_SURROGATE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct chaos_mlp chaos_mlp;

/* ensemble networks of 16 Fourier features -> width -> width -> width ->
 * outputs, SiLU; deterministic initialisation from seed. */
int chaos_mlp_create(int ensemble, int width, int outputs, uint64_t seed, int device,
                     chaos_mlp **out);
int chaos_mlp_destroy(chaos_mlp *h);
const char *chaos_mlp_last_error(void);

/* Box of the parameter plane mapped to [0, 1]^2 before the features. */
int chaos_mlp_set_domain(chaos_mlp *h, double u0, double u1, double v0, double v1);
/* The 8 frequency vectors w_f (8 x 2 floats, cycles over the unit box) of
 * the features sin / cos (2 pi w_f . (u, v)); default: (j/2, 0) and (0, j/2),
 * j = 1..4. */
int chaos_mlp_set_features(chaos_mlp *h, const float *freqs);
/* Targets are standardised with these per-output mean and std (outputs floats each). */
int chaos_mlp_set_target_scale(chaos_mlp *h, const float *mean, const float *stdev);

int64_t chaos_mlp_num_params(chaos_mlp *h);
int chaos_mlp_get_params(chaos_mlp *h, float *host);
int chaos_mlp_set_params(chaos_mlp *h, const float *host);

/* Loss gradient on rows points (device xy rows x 2, T rows x outputs
 * doubles) without an update: grads_out (host, E x params) and per-network
 * losses (host, E), either may be NULL. */
int chaos_mlp_gradient(chaos_mlp *h, const double *xy, const double *T, int64_t rows,
                       float *grads_out, float *loss_out);

/* Adam (lr, betas 0.9 / 0.999) over `steps` mini-batches of `batch` rows of
 * the N device points, seeded reshuffle per epoch; last losses to loss_out. */
int chaos_mlp_train(chaos_mlp *h, const double *xy, const double *T, int64_t N, int steps,
                    int batch, float lr, uint64_t seed, void *stream, float *loss_out);

/* Ensemble mean and std (device, N x outputs floats each, either may be NULL). */
int chaos_mlp_predict(chaos_mlp *h, const double *xy, int64_t N, float *mean, float *stdev,
                      void *stream);

#ifdef __cplusplus
}
#endif
#endif
