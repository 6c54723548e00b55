// fpho_internal.h -- host-side helpers shared by the forcepho_b200 translation units.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "fpho.h"

struct fpho_patch;

namespace fpho {

struct PatchView;
struct TileArgs;

// Record a failure message for fpho_last_error() and return `code`.
int set_error(int code, const char *fmt, ...);
void clear_error();

// Tile-kernel variants (threads per CTA x pixels per thread).
int variant_count();
int variant_tile_pixels(int v);
int variant_threads(int v);
bool variant_has_exact(int v);  // exact-residual kernels compiled for variant v
int variant_split(int v);       // 0: tile_body; NW: tile_body_split with NW warps per tile
size_t tile_smem_bytes(int variant, int live_cap, int idx_cap, int stride);
int device_sms();  // SMs of the current device (cached)
// One CTA per tile; or, with `order` and `counter` (both device pointers), the
// persistent form taking tiles in that order (see order_tiles).
// `exact` selects the exact-residual kernel (variant_has_exact must hold).
int launch_tile_kernel(int variant, const TileArgs &A, int n_tiles, cudaStream_t stream,
                       bool grad, const int *order = nullptr, int *counter = nullptr,
                       bool exact = false);

PatchView make_view(const fpho_patch *p);

// Device memory of handles (patches, batches, store scratch) comes from the
// device's default memory pool, told to keep freed memory: creating and
// freeing handles one after another then reuses pool memory instead of a
// driver allocation each time (on a busy machine those took milliseconds to
// seconds, erratically).  pool_malloc returns only once the allocation is
// usable from any stream; pool_free first waits for the device, as cudaFree
// does, so memory still read by a kernel is never reused.  The pool keeps
// the high-water mark of handle memory until the process exits.
cudaError_t pool_malloc(void **p, size_t bytes);
void pool_free(void *p);

}  // namespace fpho
