// Pipelined stepping from host buffers: pond_step_host / pond_sync.
//
// A caller whose states live in host memory (a host-side coupling code, a
// sequence of independent states) pays two PCIe copies per step.  Issued in
// order on one stream they add to the step time; here call k copies its input
// into input slot k % 2 on an upload stream, steps on the context's stream
// into output buffer k % 2 (the context's own double buffer), and reads rho
// and g back on a download stream, with events between them, so the copies
// of one call run while the neighbouring calls compute.
//
//   upload(k)   waits: step(k-2) done        (it read input slot k % 2)
//   step(k)     waits: upload(k) done, download(k-2) done (it read output k % 2)
//   download(k) waits: step(k) done
#include <cuda_runtime.h>

#include "pond_internal.h"

using namespace pond;

namespace pond {

static int pipe_setup(pond_ctx* c) {
  if (c->h2d) return POND_OK;
  const size_t bytes[3] = {(size_t)c->Q * c->N * c->elem, (size_t)c->N * c->elem, (size_t)4 * c->N * c->elem};
  void** slots[3] = {c->in_f, c->in_rho, c->in_g};
  for (int s = 0; s < 2; s++)
    for (int k = 0; k < 3; k++) {
      cudaError_t e = cudaMalloc(&slots[k][s], bytes[k]);
      if (e != cudaSuccess) {
        cudaGetLastError();
        return set_error(POND_ERR_NOMEM, "pond_step_host: input slots (%zu bytes)", bytes[0] + bytes[1] + bytes[2]);
      }
    }
  cudaError_t e = cudaStreamCreateWithFlags(&c->h2d, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->d2h, cudaStreamNonBlocking);
  for (int s = 0; s < 2 && e == cudaSuccess; s++) {
    e = cudaEventCreateWithFlags(&c->ev_in_ready[s], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_step_done[s], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_out_free[s], cudaEventDisableTiming);
  }
  return e == cudaSuccess ? POND_OK : cuda_fail(e, "pond_step_host set-up");
}

int pipe_drain(pond_ctx* c) {
  if (!c->pipe_pending) return POND_OK;
  cudaError_t e = cudaStreamSynchronize(c->h2d);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->d2h);
  if (e != cudaSuccess) return cuda_fail(e, "pond_sync");
  c->pipe_pending = false;
  return POND_OK;
}

void pipe_free(pond_ctx* c) {
  if (c->h2d) cudaStreamSynchronize(c->h2d);
  if (c->d2h) cudaStreamSynchronize(c->d2h);
  for (int s = 0; s < 2; s++) {
    cudaFree(c->in_f[s]); cudaFree(c->in_rho[s]); cudaFree(c->in_g[s]);
    c->in_f[s] = c->in_rho[s] = c->in_g[s] = nullptr;
    for (cudaEvent_t* ev : {&c->ev_in_ready[s], &c->ev_step_done[s], &c->ev_out_free[s]}) {
      if (*ev) cudaEventDestroy(*ev);
      *ev = nullptr;
    }
  }
  if (c->h2d) cudaStreamDestroy(c->h2d);
  if (c->d2h) cudaStreamDestroy(c->d2h);
  c->h2d = c->d2h = nullptr;
}

}  // namespace pond

extern "C" {

int pond_step_host(pond_ctx* c, const void* f_in, const void* rho_in, const void* g_in, void* rho_out,
                   void* g_out) {
  if (!c || !f_in || !rho_in || !g_in) return set_error(POND_ERR_ARG, "pond_step_host: null input");
  if (!c->initialized) return set_error(POND_ERR_STATE, "pond_step_host before pond_init/pond_set_state");
  if (c->p.learned) return set_error(POND_ERR_STATE, "pond_step_host runs the plain start; detach the predictor");
  if (c->p.ddf) return set_error(POND_ERR_UNSUPPORTED, "pond_step_host carries no energy populations");
  cudaSetDevice(c->p.device);
  int st = pipe_setup(c);
  if (st != POND_OK) return st;
  const int s = (int)(c->pipe_k & 1);
  const size_t bytes[3] = {(size_t)c->Q * c->N * c->elem, (size_t)c->N * c->elem, (size_t)4 * c->N * c->elem};
  const void* src[3] = {f_in, rho_in, g_in};
  void* in[3] = {c->in_f[s], c->in_rho[s], c->in_g[s]};
  // upload into slot s once the step that last read it is done
  cudaError_t e = cudaStreamWaitEvent(c->h2d, c->ev_step_done[s], 0);
  for (int k = 0; k < 3 && e == cudaSuccess; k++)
    e = cudaMemcpyAsync(in[k], src[k], bytes[k], cudaMemcpyHostToDevice, c->h2d);
  if (e == cudaSuccess) e = cudaEventRecord(c->ev_in_ready[s], c->h2d);
  // step into output buffer s once the upload is in and the read-back that last used it is done
  if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream, c->ev_in_ready[s], 0);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream, c->ev_out_free[s], 0);
  if (e != cudaSuccess) return cuda_fail(e, "pond_step_host upload");
  c->pipe_pending = true;
  void* out[3] = {c->f[s], c->rho[s], c->g[s]};
  st = launch_step_io(c, in, out);
  if (st != POND_OK) return st;
  e = cudaEventRecord(c->ev_step_done[s], c->stream);
  // read back rho and g of the result
  if (e == cudaSuccess) e = cudaStreamWaitEvent(c->d2h, c->ev_step_done[s], 0);
  if (e == cudaSuccess && rho_out) e = cudaMemcpyAsync(rho_out, out[1], bytes[1], cudaMemcpyDeviceToHost, c->d2h);
  if (e == cudaSuccess && g_out) e = cudaMemcpyAsync(g_out, out[2], bytes[2], cudaMemcpyDeviceToHost, c->d2h);
  if (e == cudaSuccess) e = cudaEventRecord(c->ev_out_free[s], c->d2h);
  if (e != cudaSuccess) return cuda_fail(e, "pond_step_host");
  c->cur = s;  // the result is the context's current state
  c->istep++;
  c->curtime += c->p.dt;
  c->have_sums = false;
  c->pipe_k++;
  return POND_OK;
}

int pond_sync(pond_ctx* c) {
  if (!c) return set_error(POND_ERR_ARG, "null context");
  cudaSetDevice(c->p.device);
  return pipe_drain(c);
}

}  // extern "C"
