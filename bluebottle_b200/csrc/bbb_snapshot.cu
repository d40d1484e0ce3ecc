/* bbb_snapshot.cu -- asynchronous output snapshots.
 *
 * The reference's output writers (out_VTK, src/vtk.c:48; cgns_flow_field
 * and cgns_particles, src/recorder.c:487-1890) read the host arrays u, v,
 * w, p, phase and parts, which the reference's loop refreshes with a
 * blocking cuda_dom_pull / cuda_part_pull before every output
 * (src/bluebottle.c:717-760): the time loop stops for the whole transfer.
 * Here bbb_snapshot_start copies those fields on the device into a
 * snapshot buffer, ordered after the step on the library's stream (a
 * device-to-device copy, a fraction of a millisecond), and moves the
 * snapshot to pinned host staging on a stream of its own, so the transfer
 * overlaps the steps that follow; bbb_snapshot_finish waits for it and
 * writes the snapshot into the host arrays for the writers.
 *
 * The buffers (a device copy and pinned host staging of the six fields)
 * are allocated by the first start and released by cuda_dom_free. */
#include "bbb_internal.h"

namespace {

struct snap_field {
  void *dev;            /* device field                     */
  void *host;           /* host array the writers read      */
  size_t bytes;
};

struct snap_state {
  int busy;                     /* started and not finished          */
  size_t bytes[6];              /* allocated sizes                   */
  void *dcopy[6];               /* device snapshot                   */
  void *hstage[6];              /* pinned host staging               */
  cudaStream_t out;             /* the transfer's stream             */
  cudaEvent_t taken, landed;    /* device copy done, host copy done  */
};

snap_state S;

/* u, v, w, p, phase, parts of the current set-up */
int snap_fields(snap_field (&f)[6])
{
  const dom_struct *d = &Dom;
  f[0] = {g_dev.u, u, sizeof(real) * (size_t)d->Gfx.s3b};
  f[1] = {g_dev.v, v, sizeof(real) * (size_t)d->Gfy.s3b};
  f[2] = {g_dev.w, w, sizeof(real) * (size_t)d->Gfz.s3b};
  f[3] = {g_dev.p, p, sizeof(real) * (size_t)d->Gcc.s3b};
  f[4] = {g_dev.phase, phase, sizeof(int) * (size_t)d->Gcc.s3b};
  f[5] = {g_dev.parts, parts,
          nparts > 0 && g_dev.np == nparts ? sizeof(part_struct) * (size_t)nparts : 0};
  return 6;
}

void snap_free_buffers(void)
{
  for(int a = 0; a < 6; a++) {
    if(S.dcopy[a]) cudaFree(S.dcopy[a]);
    if(S.hstage[a]) cudaFreeHost(S.hstage[a]);
    S.dcopy[a] = S.hstage[a] = NULL;
    S.bytes[a] = 0;
  }
}

}  // namespace

/* called by cuda_dom_free */
void bbb_snapshot_release(void)
{
  if(S.out) {
    cudaStreamSynchronize(S.out);
    cudaStreamDestroy(S.out);
    cudaEventDestroy(S.taken);
    cudaEventDestroy(S.landed);
    S.out = NULL;
  }
  snap_free_buffers();
  S.busy = 0;
}

extern "C" int bbb_snapshot_start(void)
{
  bbb_dev_require();
  if(!g_dev.ready) return BBB_ERR_STATE;
  if(S.busy) return BBB_ERR_STATE;
  snap_field f[6];
  snap_fields(f);
  if(!S.out) {
    BBB_CK(cudaStreamCreateWithFlags(&S.out, cudaStreamNonBlocking));
    BBB_CK(cudaEventCreateWithFlags(&S.taken, cudaEventDisableTiming));
    BBB_CK(cudaEventCreateWithFlags(&S.landed, cudaEventDisableTiming));
  }
  for(int a = 0; a < 6; a++) {
    if(f[a].bytes == S.bytes[a]) continue;
    if(S.dcopy[a]) cudaFree(S.dcopy[a]);
    if(S.hstage[a]) cudaFreeHost(S.hstage[a]);
    S.dcopy[a] = S.hstage[a] = NULL;
    S.bytes[a] = 0;
    if(f[a].bytes == 0) continue;
    BBB_CK(cudaMalloc(&S.dcopy[a], f[a].bytes));
    BBB_CK(cudaHostAlloc(&S.hstage[a], f[a].bytes, cudaHostAllocDefault));
    if(!S.dcopy[a] || !S.hstage[a]) { snap_free_buffers(); return BBB_ERR_CUDA; }
    S.bytes[a] = f[a].bytes;
  }
  /* the device copy, after the step, on the library's stream */
  for(int a = 0; a < 6; a++)
    if(S.bytes[a])
      BBB_CK(cudaMemcpyAsync(S.dcopy[a], f[a].dev, S.bytes[a],
        cudaMemcpyDeviceToDevice, g_dev.stream));
  BBB_CK(cudaEventRecord(S.taken, g_dev.stream));
  /* the transfer, on its own stream, once the copy is taken */
  BBB_CK(cudaStreamWaitEvent(S.out, S.taken, 0));
  for(int a = 0; a < 6; a++)
    if(S.bytes[a])
      BBB_CK(cudaMemcpyAsync(S.hstage[a], S.dcopy[a], S.bytes[a],
        cudaMemcpyDeviceToHost, S.out));
  BBB_CK(cudaEventRecord(S.landed, S.out));
  if(bbb_last_status() == BBB_ERR_CUDA) return BBB_ERR_CUDA;
  S.busy = 1;
  return BBB_OK;
}

extern "C" int bbb_snapshot_finish(void)
{
  if(!S.busy) return BBB_ERR_STATE;
  S.busy = 0;
  BBB_CK(cudaEventSynchronize(S.landed));
  if(bbb_last_status() == BBB_ERR_CUDA) return BBB_ERR_CUDA;
  snap_field f[6];
  snap_fields(f);
  for(int a = 0; a < 6; a++)
    if(S.bytes[a] && S.bytes[a] == f[a].bytes && f[a].host)
      memcpy(f[a].host, S.hstage[a], S.bytes[a]);
  return BBB_OK;
}

extern "C" int bbb_snapshot_busy(void) { return S.busy; }
