// Internal (C++) interface between the time-step library (cfdgpu.cu) and the
// learned-guess network (mpnn.cu).  Not part of the C ABI.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/cfdgpu.h"

namespace cfdgpu {

struct GraphView {
  int nNode = 0, ndof = 0, ndim = 0, nfree = 0;
  const int32_t *rowptr = nullptr;   // node graph (includes the node itself)
  const int32_t *colidx = nullptr;
  const double *coords = nullptr;    // nNode*ndim
  const uint8_t *fixmask = nullptr;  // per node, bit d = dof d prescribed
  cudaStream_t stream = nullptr;
};

// device view of a handle's mesh graph
int handle_graph(cfdgpu_handle *h, GraphView *out);

// host-side scheduling of a handle's step: blocking (sleeping) host waits,
// the number of Arnoldi steps per graph chunk (1..64) and the number of
// chunks in flight beyond the one the host waits for (1..8); results do not
// depend on any of them (Arnoldi kernels after convergence are no-ops)
int set_host_schedule(cfdgpu_handle *h, bool blocking, int chunk, int depth);

// replace the handle's stream by a non-blocking stream of the given
// priority (lower value = higher priority); cached Arnoldi graphs follow the
// priority of the stream they are launched into
int set_stream_priority(cfdgpu_handle *h, int priority);

// size of a handle's system: dofs and BSR blocks (work estimate)
int handle_work(cfdgpu_handle *h, double *dofs, double *blocks);

// guess model attached to a handle: given u_n (solnPrev after the time
// update) and u_{n-1} (solnPrev2), write the predicted increment for every
// dof into delta (device, nNode*ndof); returns 0 on success
int mpnn_predict_increment(cfdgpu_mpnn *m, const double *u_n, const double *u_nm1, double *delta, cudaStream_t s);

}  // namespace cfdgpu
