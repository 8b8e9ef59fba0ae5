/* idx2g: B200 (sm_100a) implementation of the idx2 encode/decode hot path.
 *
 * C ABI: plain pointers, sizes and integer error codes; no C++ or torch types.
 * The entry points replace the reference's library calls for this path:
 *
 *   idx2g_encode          <- idx2::Encode(idx2_file*, const params&, brick_copier&)
 *                            (Source/Core/idx2Encode.h:144, Core/idx2Encode.cpp:390)
 *                            together with the SetParams + Finalize steps of idx2App
 *                            (Source/Applications/idx2App.cpp:217, Core/idx2Common.cpp:726)
 *   idx2g_check_params    <- Finalize's validation (Core/idx2Common.cpp:726-754)
 *   idx2g_dataset_open    <- idx2::Init(idx2_file*, params&) (Source/idx2.cpp:23)
 *   idx2g_output_grid     <- idx2::GetOutputGrid (Source/idx2.cpp:36, Core/idx2Common.cpp:772)
 *   idx2g_decode          <- idx2::Decode(idx2_file*, params&, buffer*) (Source/idx2.cpp:43,
 *                            Core/idx2Decode.cpp:326) with OutMode RegularGridMem
 *   idx2g_dataset_close   <- idx2::Destroy (Source/idx2.cpp:52)
 *
 * Error codes are the reference's idx2_err_code values (Core/ErrorCodes.h:6-10 followed by
 * Core/idx2Common.h:36-56): 0 is NoError, 22 BrickSizeTooBig, 23 TooManyLevels, ...
 * Codes >= 100 belong to this library (see idx2g_error_string).
 *
 * Threading: one idx2g_ctx per host thread; all device work of a context is ordered on its
 * CUDA stream. The caller owns every buffer it passes in.
 */
#ifndef IDX2G_H
#define IDX2G_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IDX2G_API __attribute__((visibility("default")))

enum
{
  IDX2G_FLOAT32 = 0,
  IDX2G_FLOAT64 = 1
};

/* Mirrors idx2::params (Core/idx2Common.h:74-108). */
typedef struct idx2g_params
{
  /* metadata and encode parameters */
  char name[64];
  char field[64];
  int dims[3];
  int dtype;               /* IDX2G_FLOAT32 or IDX2G_FLOAT64 */
  int brick_dims[3];       /* default 32 32 32; 2D fields use 32 32 1 */
  int num_levels;          /* 0: guess as the reference does */
  double tolerance;        /* absolute tolerance of the encode */
  int bricks_per_chunk;    /* default 4096 */
  int chunks_per_file;     /* default 64 */
  int files_per_dir;       /* default 64 */
  int bit_planes_per_chunk;/* default 1 */
  int bit_planes_per_file; /* default 16 */
  int version[2];          /* 1 0 */
  char out_dir[512];       /* encode output directory (default ".") */
  /* decode parameters */
  char input_file[512];    /* path of the .idx2 metadata file */
  char in_dir[512];        /* directory holding <name>/<field>/... (default ".") */
  int has_extent;          /* 1: decode only [first, last] (inclusive) */
  int first[3];
  int last[3];
  int downsampling[3];     /* per-axis downsampling factor (power of two exponent) */
  double decode_tolerance;
} idx2g_params;

typedef struct idx2g_encode_info
{
  double kernel_ms;        /* device time of the brick kernels (CUDA events) */
  double device_s;         /* wall time of the device stage incl. copies */
  double pack_s;           /* host packing (chunks, zstd) */
  double write_s;          /* file writes */
  long long stream_bytes;  /* bit-plane stream bytes produced on the device */
  long long exp_bytes;     /* uncompressed exponent bytes */
  long long file_bytes;    /* total bytes of the written files */
  long long kernel_launches;
  double value_min, value_max;
  int num_levels;
  double level_kernel_ms[16];      /* device time of each level's launch */
  long long level_out_bytes[16];   /* stream + exponent bytes produced by each level */
} idx2g_encode_info;

typedef struct idx2g_ctx idx2g_ctx;
typedef struct idx2g_dataset idx2g_dataset;

/* Defaults of the reference's params / idx2App options. */
IDX2G_API void idx2g_params_init(idx2g_params* p);
IDX2G_API const char* idx2g_error_string(int code);
IDX2G_API const char* idx2g_version(void);

/* device: CUDA ordinal; stream: a cudaStream_t or NULL (the context creates one). */
IDX2G_API int idx2g_ctx_create(int device, void* stream, idx2g_ctx** ctx);
IDX2G_API int idx2g_ctx_destroy(idx2g_ctx* ctx);

/* Validate encode parameters exactly as Finalize does; returns the reference's code. */
IDX2G_API int idx2g_check_params(const idx2g_params* p);

/* Encode a field (x fastest, dims from p) and write <out_dir>/<name>/<field>.idx2 and the
   data files. field_on_device: 1 if field is a device pointer on the context's device. */
IDX2G_API int idx2g_encode(idx2g_ctx* ctx, const idx2g_params* p, const void* field,
                           int field_on_device, idx2g_encode_info* info);

/* The device stage of idx2g_encode alone: transform and code every brick of every level of
   a device-resident field, leaving the coded streams in the context's device workspace (no
   packing, no files). For measuring the kernels; the streams are the ones idx2g_encode packs. */
IDX2G_API int idx2g_encode_device(idx2g_ctx* ctx, const idx2g_params* p, const void* d_field,
                                  idx2g_encode_info* info);

/* Decode side (idx2.cpp:23-52). open reads the metadata file (p->input_file) and the chunk
   index of every data file and makes the compressed dataset resident on the device. */
IDX2G_API int idx2g_dataset_open(idx2g_ctx* ctx, const idx2g_params* p, idx2g_dataset** ds);
IDX2G_API int idx2g_output_grid(const idx2g_dataset* ds, const idx2g_params* p, int from3[3],
                                int dims3[3], int strd3[3]);
/* Decode into out (Prod(dims3) elements of the dataset's dtype). out_on_device: 1 if out is
   a device pointer on the context's device. */
IDX2G_API int idx2g_decode(idx2g_ctx* ctx, idx2g_dataset* ds, const idx2g_params* p, void* out,
                           size_t out_bytes, int out_on_device, double* kernel_ms);
IDX2G_API int idx2g_dataset_close(idx2g_dataset* ds);

/* Several decode requests on one dataset at once (each with its own extent, downsampling and
   tolerance, as in idx2g_decode): per level one launch over the bricks of every request that
   decodes that level, so many small region-of-interest requests fill the GPU together. The
   reference decodes one request per call (Core/idx2Decode.cpp:326 Decode). outs[i] receives
   request i's grid (out_bytes[i] at least its size); all outs are device pointers when
   out_on_device is 1, host pointers otherwise. */
IDX2G_API int idx2g_decode_batch(idx2g_ctx* ctx, idx2g_dataset* ds, const idx2g_params* p, int n,
                                 void* const* outs, const size_t* out_bytes, int out_on_device,
                                 double* kernel_ms);

/* Allocation-free decode. No counterpart in the reference: it exists for callers that cannot
   allocate device memory when they decode -- applications whose device memory belongs to
   another allocator (a framework's caching allocator, a pool sized to the whole GPU) and
   latency-bound serving loops, where cudaMalloc fails or synchronises the device. Open the
   dataset first (idx2g_dataset_open allocates the resident dataset), then call this with a
   device output buffer; it calls no cudaMalloc / cudaFree and no allocating library routine.
   Its temporaries live in a fixed device array of about 7.3 MB, taken on a device when the
   first context is created there (idx2g_ctx_create loads the library's decode kernels and
   resolves the array's device address with cudaGetSymbolAddress, that device current) and
   held until the process exits. Limits: at most 4096 bricks on the output level and, on
   each coarser level the request decodes, 8 bricks of a 3D dataset (264 of a 2D one, whose
   bricks are 33 times smaller); larger requests return ScratchTooSmall (104). The call waits for the context's stream between levels, so on a
   stream that is being captured it returns InvalidArgument. All calls share the array and it
   keeps the last call's contents (the error word is cleared by every call); calls that
   overlap on the GPU race on it. The result equals idx2g_decode's. */
IDX2G_API int idx2g_decode_noalloc(idx2g_ctx* ctx, idx2g_dataset* ds, const idx2g_params* p,
                                   void* d_out, size_t out_bytes, double* kernel_ms);

/* Brick-map decode: replaces the reference's HashMap output mode (idx2App --brick_map,
   params::out_mode::HashMap; Core/idx2Decode.cpp:446-477, Core/idx2SparseBricks.cpp:69-230).
   Decodes the whole field at p's downsampling and decode tolerance (p's extent is ignored, as
   the reference's brick map covers every brick), keeping each significant brick (a decoded
   block of a subband > 0, or of the coarsest level); every finest brick takes the finest level
   at which it or an ancestor is significant, and the file at `path` receives the reference's
   WriteBricks layout: int32 dims[3], brick dims[3], finest brick counts[3], then per finest
   brick in row-major order int32 brick[3], int32 sample dims[3] and the float64 samples (x
   fastest) of that level's brick over the finest brick's part of it. Where no brick of a
   chain is significant the reference fails; here the coarsest brick is written. */
IDX2G_API int idx2g_decode_brick_map(idx2g_ctx* ctx, idx2g_dataset* ds, const idx2g_params* p,
                                     const char* path, double* kernel_ms);

/* Batched encode: n fields (params[i], field[i]) through one device stage, then each is
   packed and written as idx2g_encode writes it (the files are identical). The reference
   encodes one field per call (Core/idx2Encode.cpp:390 Encode); here the bricks of every
   field share each level's launch, so many small or uneven fields fill the GPU together.
   flags: IDX2G_BATCH_GRAPH captures the level launches in one CUDA graph;
   IDX2G_BATCH_DEVICE_ONLY stops after the device stage (no packing, no files);
   IDX2G_BATCH_AUTOTUNE times the launch shapes once per batch signature (field count, total
   bricks, dtypes) on the context and keeps the fastest. infos may be null, else n entries;
   kernel_ms and device_s are those of the whole batch. Fields rejected by the format rules
   make the call fail with that error before any work. */
#define IDX2G_BATCH_GRAPH 1
#define IDX2G_BATCH_DEVICE_ONLY 2
#define IDX2G_BATCH_AUTOTUNE 4
IDX2G_API int idx2g_encode_batch(idx2g_ctx* ctx, const idx2g_params* params, const void* const* fields,
                                 int n, int fields_on_device, int flags, idx2g_encode_info* infos);

/* Sharded encode: one field encoded by several processes (one GPU each) into one dataset,
   the files identical to a single encode's. No counterpart in the reference, whose encode
   runs on one thread (Core/idx2Encode.cpp:390); the split follows its depth-first order
   (Core/idx2Encode.cpp:276-340): the coarsest level's bricks, in encode order, are cut into
   nshards runs and every shard codes the subtrees under its run. The coded data never moves
   between shards; they exchange only the headers of their (brick, subband) regions.

   idx2g_shard_region gives the samples shard `shard` reads ([from3, from3 + dims3)).
   idx2g_encode_shard codes that shard's bricks from d_field (a device buffer holding the
   dataset's samples [origin3, origin3 + dims3), which must cover the shard's region; origin3
   a multiple of the brick size) and returns its header payload (valid until the shard's
   finish call on the same context) and the value range of its samples. The caller exchanges
   the payloads (all-gather) and reduces the value range, then every shard calls
   idx2g_encode_shard_finish with all payloads in shard order: each writes its bricks' bytes
   into the shared data files at offsets every shard computes alike, shard 0 also the chunk
   headers, tables, exponent chunks and the metadata file. The files are complete once every
   shard's finish call has returned. flags IDX2G_SHARD_DEVICE_ONLY: the device stage alone
   (the streams stay in the context's device workspace, as idx2g_encode_device leaves them; no
   payload, no finish call). */
#define IDX2G_SHARD_DEVICE_ONLY 1
IDX2G_API int idx2g_shard_region(const idx2g_params* p, int shard, int nshards, int from3[3], int dims3[3]);
IDX2G_API int idx2g_encode_shard(idx2g_ctx* ctx, const idx2g_params* p, const void* d_field, const int origin3[3],
                                 const int dims3[3], int shard, int nshards, int flags, const void** headers,
                                 size_t* header_bytes, double* vmin, double* vmax, idx2g_encode_info* info);
IDX2G_API int idx2g_encode_shard_finish(idx2g_ctx* ctx, const idx2g_params* p, int shard, int nshards,
                                        const void* const* headers, const size_t* header_bytes, double vmin,
                                        double vmax, idx2g_encode_info* info);

/* Differentiable decode. The reference has no counterpart: its decode is integer end to end
   (Core/idx2Decode.cpp:141-320). Here the decode is also available as a real-valued linear
   operator D from the dequantised zfp-domain coefficients to the grid: the reference's decode
   with the integer inverse zfp (Core/Zfp.h:181) replaced by its real form (exact halvings in
   place of the shifts), then de-normalisation, the inverse CDF5/3 and the parent hand-off per
   level. D and its adjoint let gradients of a loss on the decoded grid reach the coefficients.

   Coefficient tensor of one field (format given by p: dims, dtype, brick dims, levels): levels
   0 (finest) to L-1; on each level the bricks in row-major order of their coordinates (x
   fastest); each brick 33^3 values (33^2 for 2D) indexed (z*33 + y)*33 + x, every coefficient
   at the position of the sample its block transforms; idx2g_coeff_count gives its length.
   Batched calls take nbatch tensors (and grids) back to back. Values are of p's dtype.
   D(idx2g_coeffs(...)) equals idx2g_decode's grid up to the floors of the integer inverse
   zfp, except in 2D where a low-band block below the coarsest level had no bit plane above
   the decode tolerance: the decode keeps the parent's values there, D writes the block's
   (zero) coefficients. */
IDX2G_API long long idx2g_coeff_count(const idx2g_params* p);
/* The dataset's dequantised coefficients (at p's decode tolerance) into d_coeffs. */
IDX2G_API int idx2g_coeffs(idx2g_ctx* ctx, idx2g_dataset* ds, const idx2g_params* p, void* d_coeffs,
                           size_t bytes, double* kernel_ms);
/* grid = D(coefficients) for nbatch fields (device pointers). */
IDX2G_API int idx2g_synth(idx2g_ctx* ctx, const idx2g_params* p, int nbatch, const void* d_coeffs,
                          void* d_grid, double* kernel_ms);
/* coefficient gradient = D^T(grid gradient) for nbatch fields (device pointers). */
IDX2G_API int idx2g_synth_adjoint(idx2g_ctx* ctx, const idx2g_params* p, int nbatch,
                                  const void* d_grid_grad, void* d_coeff_grad, double* kernel_ms);

/* Number of kernels this library has launched on the context so far (a diagnostic for
   benchmarks; no counterpart in the reference). */
IDX2G_API long long idx2g_ctx_launches(const idx2g_ctx* ctx);

/* Metadata of an open dataset (the fields of the .idx2 file): name and field (64 bytes
   each, NUL-terminated), dims, dtype, number of levels, encode tolerance, and the bytes
   the dataset keeps resident on the device. */
IDX2G_API int idx2g_dataset_info(const idx2g_dataset* ds, char* name, char* field, int dims3[3],
                                 int* dtype, int* num_levels, double* tolerance,
                                 long long* resident_bytes);

#ifdef __cplusplus
}
#endif

#endif
