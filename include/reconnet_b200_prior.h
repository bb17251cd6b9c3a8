/* reconnet_b200 prior-solver shim: the total-variation entry points of the
 * reference's prior-solver library (PriorFunctionSolver/TVSQS.cu), with the
 * same names and signatures, for callers that load that library
 * (python/PriorFunctionSolver2.py:161-205).  They are exported by
 * libreconnet_b200_prior.so, a thin forwarder to rn_tv_iso_sqs_host in
 * libreconnet_b200.so (the reference's ReconNet4D library exports a different
 * cTVSQS2D, so the two cannot share one library).
 *
 * Host pointers, synchronous; arrays are [nb][nx][ny][nc] (2D) and
 * [nb][nx][ny][nz][nc] (3D), C order.  s1 / s2 are the first / second
 * derivatives of the isotropic TV surrogate, var the local variation
 * sqrt(|backward gradient|^2 + eps).  On error the outputs are untouched and
 * rn_last_error() of libreconnet_b200 says why. */
#ifndef RECONNET_B200_PRIOR_H
#define RECONNET_B200_PRIOR_H

#ifdef __cplusplus
extern "C" {
#endif

/* replaces PriorFunctionSolver/TVSQS.cu:101-146 */
void cTVSQS2D(float* s1, float* s2, float* var, const float* img, int nb, int nx, int ny, int nc, float eps);

/* replaces PriorFunctionSolver/TVSQS.cu:291-345 */
void cTVSQS3D(float* s1, float* s2, float* var, const float* img, int nb, int nx, int ny, int nz, int nc, float eps);

#ifdef __cplusplus
}
#endif

#endif
