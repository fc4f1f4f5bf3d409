// umma_dft.cu -- tcgen05 (5th-generation tensor core) DFT and adjoint
// contractions. Placeholder until the tensor path lands: every entry point
// reports GPAIR_ERR_STATE so that a request for a tensor precision fails
// loudly instead of silently running the CUDA-core path.
#include "gpair_internal.cuh"

int gp_tc_prepare(gpair_ctx *c)
{
    snprintf(c->last_error, sizeof(c->last_error), "tensor-core precision modes are not built in this library");
    return GPAIR_ERR_STATE;
}
int gp_tc_forward(gpair_ctx *c, int) { return gp_tc_prepare(c); }
int gp_tc_adjoint(gpair_ctx *c, int) { return gp_tc_prepare(c); }
void gp_tc_free(gpair_ctx *) {}
double gp_adjoint_scale(gpair_ctx *) { return 1.0; }
