// ftb_internal.h -- accessors shared by the library's translation units (not part of the
// C ABI): the scene's device view, the error text and the fixed-point conventions.
#pragma once
#include <stdint.h>
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/ftb200.h"
#include "ftb_layout.h"

namespace ftb {
// The device view of a scene and where it lives; false for a null scene.
bool scene_internals(const ftb_scene* s, DevScene* dev, int* device, int* sms, double* power);
// The checks every render entry point applies to its arguments (null pointers, camera
// resolution, photon count, bounce cap, film format, wavelength policy, emitted power);
// FTB_OK or the error, with its text set.
ftb_status check_render_params(const ftb_scene* s, const ftb_camera* cam, const ftb_render_params* p);
// Device residency for the render server (ftb_scene_evict / ftb_scene_restore without
// their device-wide waits): evict frees the scene's tables, stream-ordered on `stream` where
// they came from a restore (the caller guarantees no render of the scene is in flight);
// restore uploads them again with stream-ordered allocations and copies on `stream`.
ftb_status scene_evict(const ftb_scene* s, cudaStream_t stream);
ftb_status scene_restore(const ftb_scene* s, cudaStream_t stream);
bool scene_resident(const ftb_scene* s);
bool scene_evictable(const ftb_scene* s);
// Device bytes of the scene's tables (ftb_footprint.scene_bytes).
uint64_t scene_device_bytes(const ftb_scene* s);
// The mutex the scene's device engine holds while a render of it is being issued.
std::mutex& scene_mutex(const ftb_scene* s);
// The text ftb_last_error() returns (thread-local).
void set_last_error(const std::string& m);
// The default film format for an n-photon render: 62 - ceil(log2 n) - 20 in [4, 40].
int default_frac_bits(int64_t n);
// The camera as the kernels read it.
DevCam camera_to_dev(const ftb_camera* c);
// Five fixed-point tallies (32 fraction bits per unit of `power`) as an energy report.
void energy_from_tally(const unsigned long long* fx, double power, ftb_energy* e);
}  // namespace ftb
