/* dem_surrogate.h -- C ABI of the calibration surrogate: a multilayer
 * perceptron mapping contact parameters to bulk responses of a granular heap,
 * trained on the GPU from batched DEM runs (libdem_surrogate.so).
 *
 * It has no counterpart in the reference: the reference calibrates by
 * sequential Monte Carlo over plain DEM runs (Drivers/Calibration/py/smc.py,
 * Drivers/Calibration/CalibrationHeap.cpp). Here the network proposes
 * candidate parameters and batched DEM (include/dem_b200.h) judges them.
 *
 * Network: 4 inputs (sliding friction, rolling friction, restitution, PSD
 * width), 3 hidden layers of 256 with GELU (0.5 z (1 + erf(z / sqrt 2))),
 * 3 outputs (angle of repose, packing fraction, settle time). Inputs and
 * outputs are normalised with (value - mean) / std. Weights and activations
 * are BF16, products accumulate in FP32 on the tensor cores, the master
 * weights and Adam moments are FP32. Loss: mean squared error over the batch
 * and the 3 normalised outputs.
 *
 * Flat FP32 parameter vector (DEM_MLP_NPARAMS floats), row-major [out][in]:
 *   W1[256][4] b1[256] W2[256][256] b2[256] W3[256][256] b3[256] W4[3][256] b4[3]
 */
#ifndef DEM_SURROGATE_H
#define DEM_SURROGATE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DEM_MLP_INPUTS  4
#define DEM_MLP_HIDDEN  256
#define DEM_MLP_OUTPUTS 3
#define DEM_MLP_NPARAMS 133635

#define DEM_MLP_OK            0
#define DEM_MLP_ERR_BAD_INPUT 4
#define DEM_MLP_ERR_CUDA      5
#define DEM_MLP_ERR_TIMEOUT   2  /* a tensor-core wait ran out (device status) */

typedef struct dem_mlp dem_mlp;

/* Network on `device` for batches of up to `capacity` rows; weights drawn
 * He-uniform from `seed`, biases zero, normalisation the identity. */
int  dem_mlp_create(int device, int capacity, uint64_t seed, dem_mlp **out);
/* in_mean[4], in_std[4], out_mean[3], out_std[3]. */
int  dem_mlp_set_normalisation(dem_mlp *h, const float *in_mean, const float *in_std, const float *out_mean,
                               const float *out_std);
int  dem_mlp_get_params(dem_mlp *h, float *params);
int  dem_mlp_set_params(dem_mlp *h, const float *params);
/* y[n][3] (raw units) for x[n][4] (raw units); host arrays. */
int  dem_mlp_forward(dem_mlp *h, const float *x, int n, float *y);
/* Loss and gradient (DEM_MLP_NPARAMS floats) of the batch, no update. */
int  dem_mlp_gradients(dem_mlp *h, const float *x, const float *t, int n, float *loss, float *grads);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on the batch; *loss is the
 * batch loss before the update. */
int  dem_mlp_train_step(dem_mlp *h, const float *x, const float *t, int n, float lr, float *loss);
/* Device time of the forward pass (inputs already on the device from the
 * last call) for n rows, averaged over reps launches: *ms per pass. */
int  dem_mlp_time_forward(dem_mlp *h, int n, int reps, float *ms);
const char *dem_mlp_last_error(dem_mlp *h);
void dem_mlp_destroy(dem_mlp *h);

#ifdef __cplusplus
}
#endif
#endif
