// Decode side: dataset index (host parse of the data files, device-resident copy of
// the chunk payloads) and the level-by-level device decode (Core/idx2Decode.cpp:326).
#pragma once

#include "device.h"
#include "format.h"

namespace idx2g
{

struct dataset_handle;
struct decode_request;

// Plan a decode request on the host (ROI, downsampling masks, tolerance, per-level brick
// lists); need_bytes is the size of the output grid.
int plan_decode(const dataset_handle* ds, const params& p, decode_request* rq, size_t* need_bytes);

int dataset_open(device_ctx* ctx, const params& p, dataset_handle** out);
int dataset_output_grid(const dataset_handle* ds, const params& p, grid* g);
int dataset_decode(device_ctx* ctx, dataset_handle* ds, const params& p, void* out, size_t out_bytes,
                   bool out_on_device, double* kernel_ms);
// Several requests at once (one launch per level over all of their bricks).
int dataset_decode_batch(device_ctx* ctx, dataset_handle* ds, const params* ps, int n, void* const* outs,
                         const size_t* out_bytes, bool out_on_device, double* kernel_ms);
// The dequantised coefficients of the whole dataset (decode tolerance of p) into d_coeffs.
int dataset_decode_brick_map(device_ctx* ctx, dataset_handle* ds, const params& p, const char* path,
                             double* kernel_ms);
int dataset_coeffs(device_ctx* ctx, dataset_handle* ds, const params& p, void* d_coeffs, size_t bytes,
                   double* kernel_ms);
void dataset_close(dataset_handle* ds);

// Differentiable decode (adjoint.cu): elements of one field's coefficient tensor, and the
// real-valued decode operator (adjoint = false: coefficients -> grid) or its adjoint (grid
// gradient -> coefficient gradient) on nbatch fields of format f.
long long synth_coeff_count(const dataset_format& f);
int synth(device_ctx* ctx, const dataset_format& f, int nbatch, const void* d_in, void* d_out, bool adjoint,
          double* kernel_ms);
// Allocation-free variant of dataset_decode (device output only; see decode.cu).
int dataset_decode_noalloc(device_ctx* ctx, dataset_handle* ds, const params& p, void* d_out,
                           size_t out_bytes, double* kernel_ms);
const dataset_format& dataset_fmt(const dataset_handle* ds);
size_t dataset_resident_bytes(const dataset_handle* ds);

} // namespace idx2g
