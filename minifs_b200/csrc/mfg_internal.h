// Host-side layout of objects shared by the library's translation units.
#pragma once

#include <cstdint>
#include <vector>

#include "mfgpu.h"

// Device-resident preprocessing of one raw grid (mfg_prep_gpu_run): the
// raw arrays, the lists built from them and every output, all in device
// memory of `device`.
struct mfg_prep_gpu {
  int32_t device = 0;
  int32_t N = 0, F = 0, C = 0, B = 0;
  int64_t n = 0;   // C + B
  int32_t L = 0;   // face-node positions
  int32_t LB = 0;  // of the boundary faces
  int32_t S = 0;   // cell-face slots
  int32_t K = 0;   // c2n entries
  double kernel_ms = 0.0;
  std::vector<void *> allocs;
  double *x = nullptr, *y = nullptr, *z = nullptr;
  int32_t *nnpf = nullptr, *f2n = nullptr, *f2c = nullptr, *bctype = nullptr;
  int32_t *fptr = nullptr, *cptr = nullptr, *cf = nullptr;
  double *xfn = nullptr, *yfn = nullptr, *zfn = nullptr, *area = nullptr;
  double *xfc = nullptr, *yfc = nullptr, *zfc = nullptr;
  double *xcc = nullptr, *ycc = nullptr, *zcc = nullptr, *vol = nullptr;
  int32_t *c2n_ptr = nullptr, *c2n = nullptr, *c2n_cell = nullptr, *nnpc = nullptr;
  int32_t *nbptr = nullptr, *nblist = nullptr, *bent_face = nullptr;
  int32_t *ncptr = nullptr, *nclist = nullptr;
  double *wnode = nullptr, *wbface = nullptr, *wc2n = nullptr;
  int32_t *nmark = nullptr, *nodesymm = nullptr;
  double *xsym = nullptr, *ysym = nullptr, *zsym = nullptr;
};
