// Single translation unit for libgromos_nb.so: kernel templates and their
// launch sites are compiled together (whole-program CUDA compilation).
#include "pairlist.cu"
#include "forces.cu"
#include "water.cu"
#include "water_ps.cu"
#include "api.cu"
#include "md.cu"
#include "batch.cu"
#include "server.cu"
#include "frames.cu"
#include "noalloc.cu"
