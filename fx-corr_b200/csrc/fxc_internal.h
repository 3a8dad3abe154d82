// fxc_internal.h — library-internal entry points shared by the host-side
// translation units (api.cu, noalloc.cu, serve.cu).  Not part of the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "fxc.h"

namespace fxc {

// Records msg as the calling thread's last error and returns s.
fxc_status internal_fail(fxc_status s, const char* msg);

// The failure-injection settings of fxc_debug_inject_wait_timeout, copied into
// the kernel parameters of every correlation launch (0, 0 in normal use).
void internal_debug_settings(uint32_t* wait_polls, uint32_t* debug_flags);

// Maps a device error word (ERR_*) to a status and message; FXC_OK for 0.
fxc_status internal_device_error(uint32_t err);

// Validates c and fills the host copies of the decode tables: byte LUTs of
// both shuffles, f32 levels, the per-station exact level scales and shuffle kinds.
fxc_status internal_prepare_tables(const fxc_scan_cfg* c, uint32_t* lut2048, float* lv512,
                                   float scale[2], int kind[2]);

// (Re)binds an idle scan to cfg, reusing its device buffers (grown and
// charged to the engine's HBM budget where cfg needs more).
fxc_status scan_bind(fxc_scan* s, const fxc_scan_cfg* cfg);

struct BatchScan;

int engine_sm_count(const fxc_engine* e);
int engine_device(const fxc_engine* e);
fxc_engine* scan_engine(const fxc_scan* s);
// Charges / returns bytes of the engine's HBM budget (FXC_EBUSY when over).
fxc_status engine_reserve(fxc_engine* e, uint64_t bytes);
void engine_release(fxc_engine* e, uint64_t bytes);

// Describes one sector of scan s on device inputs for a batch (*group = its
// batch group), or leaves *group = -1 when the sector takes the per-scan
// path (empty sector, both correlation and phased products, phased above FFT
// 8192, correlation above 16384, odd band shift at 16384).  d_raw_out receives
// the phased .raw frames of a scan with FXC_PROD_RAW.  Grows the scan's
// frame-record buffer; launches nothing.
fxc_status batch_describe(fxc_scan* s, const uint8_t* r1, const uint8_t* r2, uint64_t nf,
                          uint64_t first, double* d_acc, uint8_t* d_raw_out, BatchScan* out,
                          int* group);
// The per-scan sector path (fxc_sector_run_device).
fxc_status run_sector_internal(fxc_scan* s, const uint8_t* r1, const uint8_t* r2, uint64_t nf,
                               uint64_t first, double* d_acc, uint8_t* d_raw_out,
                               cudaStream_t st);

// A sector copied into one of its scan's sector slots, for another stream to
// compute (the serving loop's batches).
struct StagedSector {
  uint32_t slot;
  const uint8_t* d_raw1;
  const uint8_t* d_raw2;
  double* d_acc;      // 5 * H doubles, written by the computing stream
  uint8_t* d_raw_out; // phased .raw frames (scans with FXC_PROD_RAW), else NULL
  cudaEvent_t h2d;    // after the input copies
};
// Reserves a sector slot of s and enqueues the copies of the host inputs on
// the scan's copy stream.
fxc_status sector_stage(fxc_scan* s, const uint8_t* raw1, uint64_t n1, const uint8_t* raw2,
                        uint64_t n2, uint64_t nf, StagedSector* out);
// After the sector's products were enqueued (event `computed`): the
// device-to-host copies on the scan's stream; *sector_id is then waited for
// with fxc_sector_wait.
fxc_status sector_collect(fxc_scan* s, const StagedSector& ss, cudaEvent_t computed,
                          uint64_t* sector_id);
// Gives back a staged slot whose sector was never computed.
void sector_release(fxc_scan* s, const StagedSector& ss);

// Frees a batch's device tables and partials (and their budget charge) once
// its last call's work is done; the next call grows them again.
void batch_release(fxc_batch* b);

// Registers (add) or forgets a batch, destroyed by fxc_engine_destroy.
void engine_track_batch(fxc_engine* e, fxc_batch* b, bool add);

// Registers (add) or forgets a server, so that fxc_engine_destroy can
// destroy the engine's live servers before it closes their scans.
void engine_track_server(fxc_engine* e, fxc_server* sv, bool add);

}  // namespace fxc
