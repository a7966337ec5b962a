// Camera frames on the device: the preprocessing of the reconstruction
// driver (main_sparse_inverse.cu:106-124) from raw 8/16-bit samples straight
// into a context's hologram, and background generation
// (main_create_background.cu) over a frame sequence.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

#include "../../include/rihvr.h"

namespace rihvr {

// Device buffers for one context's frame uploads, grown on first use.
struct FrameWorkspace;
void frame_workspace_free(FrameWorkspace* ws);

// Preprocess a W0 x H0 frame of `bits`-bit samples (8, 16, or 32 = floats
// holding sample values) into a W x H hologram in the workspace (*out), on
// stream st: /255, I/mean - 1 or background division, crop, zero padding of
// `pad`.  The result equals rihvr_preprocess's bit for bit.  Returns a status
// and sets the message; nothing outside the workspace is written.
int frame_to_hologram(FrameWorkspace** ws, const void* frame, int bits, int W0, int H0, const void* background,
                      const rihvr_file_params* files, int pad, int W, int H, int is_device, cudaStream_t st,
                      const float** out, long long* launches);

}  // namespace rihvr
