// libreconnet_b200_prior.so: the reference prior-solver library's total
// variation entry points (PriorFunctionSolver/TVSQS.cu:101-146, :291-345),
// forwarded to the isotropic TV surrogate of libreconnet_b200.so.
// (reconnet_b200.h is not included: its cTVSQS2D, the ReconNet4D one, has
// another signature)
#include "../../include/reconnet_b200_prior.h"

extern "C" {

int rn_tv_iso_sqs_host(float* s1, float* s2, float* var, const float* img, int nb, int nx, int ny, int nz, int nc,
                       float eps, int ndim);

void cTVSQS2D(float* s1, float* s2, float* var, const float* img, int nb, int nx, int ny, int nc, float eps) {
    rn_tv_iso_sqs_host(s1, s2, var, img, nb, nx, ny, 1, nc, eps, 2);
}

void cTVSQS3D(float* s1, float* s2, float* var, const float* img, int nb, int nx, int ny, int nz, int nc,
              float eps) {
    rn_tv_iso_sqs_host(s1, s2, var, img, nb, nx, ny, nz, nc, eps, 3);
}

}  // extern "C"
