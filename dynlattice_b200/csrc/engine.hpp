// Device data layout of one rod lattice and the host-side kernel entry points.
// All arrays live in HBM, engine-owned.  The layout itself (comments below)
// is defined in devtypes.cuh.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "devtypes.cuh"

namespace dl {

// Entry points of one compiled variant of the step kernels: the
// ahead-of-time build (interpreted yield function) or a runtime-compiled
// module with the yield function generated as code.
struct KernelSet {
  // plain variant (no contact, plates, adjoint tape or group output) ...
  const void *persistent = nullptr;
  const void *persistent1 = nullptr;  // ... its launches of one step (every step an energy step)
  const void *element = nullptr;
  const void *node = nullptr;
  // ... and the variant with those extensions
  const void *persistent_x = nullptr;
  const void *element_x = nullptr;
  const void *node_x = nullptr;
  const void *internal_force = nullptr;
  const void *gather = nullptr;
  const void *milne = nullptr;  // MilneDevice predictor-corrector (milne.cuh)
  int full_threads = 256;    // threads of a full persistent block (PersistShape) ...
  int full_threads_x = 256;  // ... and of the extended variant
  int persist_blocks = 0;    // co-resident blocks of full_threads threads
  int persist_cap[4] = {0, 0, 0, 0};    // co-resident blocks of 32, 64, 128, full_threads threads
  int persist_cap1[4] = {0, 0, 0, 0};   // the same for the one-step kernel
  int persist_cap_x[4] = {0, 0, 0, 0};  // the same for the extended variant
  int milne_cap[4] = {0, 0, 0, 0};      // the same for the predictor-corrector
  int tpb_override = 0;      // threads per block of the persistent launch (0: threads_for)
  bool jit = false;
};

// Threads per block of a launch over `work` items: 256, halved (down to 32)
// while the grid would not cover every SM -- small models then spread over
// more SMs, so each warp gets more of its SM's issue slots.
int threads_for(int work);

// Entry points of the two reverse-step kernels (adjoint_kernels.cuh).
struct AdjKernels {
  const void *node = nullptr;
  const void *elem = nullptr;
};

// adjoint.cu: the ahead-of-time build for elastic lattices
template <class T>
AdjKernels aot_adj_kernels();

// kernels.cu
template <class T>
KernelSet aot_kernels(bool plastic);
int cooperative_blocks(const void *kernel, int threads);
// fills ks.persist_blocks and ks.persist_cap
void set_persistent_caps(KernelSet &ks);
template <class T>
cudaError_t launch_steps(const KernelSet &ks, const DevModel<T> &m, const SampleSpec &smp, const StepCtx &c,
                         int mode, GridBarrier *bar, cudaStream_t s);
template <class T>
cudaError_t launch_internal_force(const KernelSet &ks, const DevModel<T> &m, double *fint, cudaStream_t s);
// One persistent launch of the predictor-corrector over c.nsteps accepted
// steps; the grid (blocks) is fixed by the caller, who sized md.partial for it.
template <class T>
cudaError_t launch_milne(const KernelSet &ks, const DevModel<T> &m, const SampleSpec &smp, const StepCtx &c,
                         GridBarrier *bar, const MilneDev<T> &md, int blocks, int tpb, cudaStream_t s);
// Element table at the current state: kind 0 strain, 1 stress, 2 plastic
// strain; material frame or spatial; out [E][6] internal element order.
template <class T>
cudaError_t launch_elem_table(const DevModel<T> &m, int kind, bool spatial, double *out, cudaStream_t s);
// blocks and threads per block of the predictor-corrector launch for a model
void milne_shape(const KernelSet &ks, int work, int *blocks, int *tpb);
// Accumulate the per-step external work of a launch into the running total,
// the sample records and the launch's energy slot; clears wstep.
cudaError_t launch_finish_wext(double *wstep, int n, double *wext_total, const SampleSpec &smp,
                               int64_t step0, int64_t sample_base, double *last_energy, cudaStream_t s);

cudaError_t launch_state_out(const double4 *pos, const double4 *rot, const double *vel, const double *X0,
                             const int32_t *node_old, int N, double *u, double *th, double *v, cudaStream_t s);
cudaError_t launch_state_in(double4 *pos, double4 *rot, double *vel, const double *X0, const int32_t *node_old,
                            int N, const double *u, const double *th, const double *v, cudaStream_t s);

enum ExecMode { EXEC_PERSISTENT = 0, EXEC_STREAM = 1, EXEC_GRAPH = 2 };

}  // namespace dl
