// fxc_internal.h — library-internal entry points shared by the host-side
// translation units (api.cu, noalloc.cu, serve.cu).  Not part of the C ABI.
#pragma once

#include <stdint.h>

#include "fxc.h"

namespace fxc {

// Records msg as the calling thread's last error and returns s.
fxc_status internal_fail(fxc_status s, const char* msg);

// Validates c and fills the host copies of the decode tables: byte LUTs of
// both shuffles, f32 levels, the per-station exact level scales and shuffle kinds.
fxc_status internal_prepare_tables(const fxc_scan_cfg* c, uint32_t* lut2048, float* lv512,
                                   float scale[2], int kind[2]);

// (Re)binds an idle scan to cfg, reusing its device buffers (grown and
// charged to the engine's HBM budget where cfg needs more).
fxc_status scan_bind(fxc_scan* s, const fxc_scan_cfg* cfg);

// Registers (add) or forgets a server, so that fxc_engine_destroy can
// destroy the engine's live servers before it closes their scans.
void engine_track_server(fxc_engine* e, fxc_server* sv, bool add);

}  // namespace fxc
