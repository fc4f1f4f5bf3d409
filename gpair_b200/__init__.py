"""gpair_b200 -- B200 (sm_100a) implementation of GPAIR's image-reconstruction
hot path: image -> DFT visibilities -> V2 / bispectrum -> chi2 + Gull-Skilling
entropy -> analytic gradients -> nonlinear CG with strong-Wolfe line search.

The compute runs in libgpair_b200.so (CUDA kernels + C ABI, include/gpair_b200.h);
this package holds the ctypes mirror of that ABI (api), OIFITS tables (oifits),
the seeded synthetic data generator (synth) and the build script (build).
"""
from .api import (IMG_CURR, IMG_TEMP, LS_BATCH, LS_TRIALS, LS_WOLFE, PREC_FP32, PREC_SPLIT16,  # noqa: F401
                  PREC_TF32, PREC_TF32X3, PREC_SPLIT16F8, REG_GULL_SKILLING, REG_L2, GpairError, Indexed, Problem, Reconstructor, cg_many, dft_tables, index_oifits, init_data, lib, problem_from_oifits, set_model,
                  workload_problem)
