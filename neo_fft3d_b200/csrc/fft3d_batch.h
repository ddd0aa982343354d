// Engine-side interface of the batched multi-plane scheduler (fft3d_batch.cu).
#pragma once
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "fft3d_b200.h"
#include "fft3d_kernels.cuh"

namespace fft3d {

// Launches and device copies of one output frame of one plane, recorded in
// issue order by phase instead of being issued.
struct Deferred {
  struct Fwd { ForwardArgs a; int bytes; int plane; };
  struct Inv { InverseArgs a; int mode; int plane; };
  struct Ola { OlaArgs a; int bytes; int plane; };
  struct Copy { void* dst; size_t dpitch; const void* src; size_t spitch; size_t width; size_t height; int plane; };
  // consecutive filter/inverse records of one plane and mode (a frame group's
  // run) merged into one work list: one CTA per block for all its frames
  struct Run { GroupRun r; int mode; int plane; };
  int plane = 0;  // index of the plane being planned (tags the records)
  std::vector<Fwd> fwd;
  std::vector<Inv> inv;
  std::vector<Ola> ola;
  std::vector<Copy> copies;  // device-to-device, before the overlap-add phase
  std::vector<Run> runs;
  std::vector<char> inv_in_run;  // per inv record: covered by a run
};

// Consecutive output frames n0 .. n0 + count - 1 of one plane planned into
// one step (Wiener/sharpen planes only: Kalman state runs frame to frame).
struct FrameGroup {
  int n0, count;
  int reverse;  // CTA order shared by the group's frames
};

// Runs plane P's per-frame control for output frame n (device buffers) with
// every launch and copy recorded in d; the spectrum-ring bookkeeping is done
// as if they had been issued. With a frame group, n is one of its frames:
// its time-domain buffer is the group's k-th, and every spectrum the group
// needs stays in the ring (grown as needed). The caller holds
// plane_mutex(P) until the recorded work is queued.
int plane_plan(fft3d_plane* P, int n, const void* const src[5], const int stride[5], void* dst, int dst_stride,
               cudaStream_t st, Deferred* d, const FrameGroup* grp = nullptr);
int plane_bt(const fft3d_plane* P);
// Forgets the spectra whose forward transforms d recorded for P (planning
// failed, so they will not run).
void plane_discard(fft3d_plane* P, const Deferred& d);
// Records that P's work so far is queued on st (fft3d_plane_reset waits for it).
void plane_mark_work(fft3d_plane* P, cudaStream_t st);
std::mutex& plane_mutex(fft3d_plane* P);
int plane_device(const fft3d_plane* P);
// Empty when the scheduler can take the plane, else the reason.
std::string plane_batchable(const fft3d_plane* P);
void count_launches(uint64_t n);
int engine_fail(int code, const std::string& msg);

}  // namespace fft3d
