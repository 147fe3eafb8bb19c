// Single translation unit of the engine: the device constants (binomial table, diagonal
// integrals) and __device__ helpers are shared by all kernels without relocatable device code.
#include "strings.cu"
#include "sigma.cu"
#include "sigma_tc.cu"
#include "sigma_same_tc.cu"
#include "davidson.cu"
#include "rdms.cu"
#include "rdms3.cu"
#include "capi.cu"
#include "mlp.cu"
#include "batch.cu"
#include "noalloc.cu"
#include "csf.cu"
