// avism_all.cu -- single translation unit of the library (kernels of one stage
// are shared by the next without relocatable device code).
#include "ctx.cu"
#include "knn.cu"
#include "sph.cu"
#include "proposal.cu"
#include "fields.cu"
#include "indexx.cu"
#include "voidfind.cu"
#include "post.cu"
#include "capi.cu"
#include "noalloc.cu"
