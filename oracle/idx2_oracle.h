/* CPU restatement of the idx2 brick codec (TEST INFRASTRUCTURE ONLY).
 *
 * This is the oracle the CUDA library is checked against. It restates, in plain
 * C, the reference's per-brick arithmetic: CDF5/3 lifting with extrapolation,
 * subband normalisation, per-block exponent + quantisation, the zfp 4^d
 * transform, the negabinary shuffle and the bit-plane group-test coder.  Each
 * function names the reference file:line it follows (paths relative to the
 * reference's Source/ directory).  It is pinned against the compiled reference
 * (oracle/_ref) by the golden vectors under tests/golden/.
 *
 * Only tests/, the smoke check and bench.py's CPU-baseline leg may load it.
 */
#ifndef IDX2_ORACLE_H
#define IDX2_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Brick geometry: 3D bricks are 33x33x33 doubles (32^3 + one extrapolated
   sample per axis), 2D bricks 33x33x1. x is the fastest axis. */
#define ORACLE_BRICK_EXT 33

/* Forward brick transform as done per brick by the encoder
   (Core/idx2Encode.cpp:291-295): extrapolation round trip on the valid dims,
   then one level of CDF5/3 with subband normalisation. */
void oracle_brick_forward(double* brick, int is2d, const int valid3[3], int level, int coarsest);

/* Only the extrapolation round trip (Core/Wavelet.cpp:68). */
void oracle_brick_extrapolate(double* brick, int is2d, const int valid3[3]);

/* Inverse brick transform (Core/idx2Decode.cpp:316-317 -> Core/Wavelet.cpp:144). */
void oracle_brick_inverse(double* brick, int is2d, int level, int coarsest);

/* Copy a child brick's low subband (16^3 non-extrapolated, stride 2) into its
   parent at local position pos3*16 (Core/idx2Encode.cpp:324-328). */
void oracle_copy_to_parent(const double* child, double* parent, int is2d, const int pos3[3]);

/* Encode the subbands of one transformed brick (Core/idx2Encode.cpp:141-272).
   Output record, appended to out (returns the byte count, or -needed if cap is
   too small):
     for each subband sb:
       int32 nblocks; int16 exps[nblocks]           (coded blocks, Morton order)
       int32 nchannels; then per channel, in first-touch order:
         int32 bpkey; int32 first_block; int32 last_block; int32 nbytes; uint8 bytes[nbytes]
   nbytes is the channel's byte-aligned block stream for this brick. */
long oracle_encode_brick(const double* brick, int is2d, int level, int nlevels, int is_f32,
                         double tol, int bpc, uint8_t* out, long cap);

/* Decode the subbands selected by mask into a zeroed (or parent-filled) brick,
   mirroring DecodeSubband (Core/idx2Decode.cpp:86-234). rec has the layout
   produced by oracle_encode_brick. spacing: per subband decode spacing
   (3 ints each, 1 = every block). Returns 0 on success. */
int oracle_decode_brick(double* brick, int is2d, int level, int nlevels, int is_f32,
                        double tol, int bpc, int mask, const int* spacing,
                        const uint8_t* rec, long rec_bytes);

/* Copy the parent's low-subband block back into a child brick
   (Core/idx2Decode.cpp:285-293). */
void oracle_copy_from_parent(const double* parent, double* child, int is2d, const int pos3[3]);

/* Block-level pieces, for known-answer tests. */
int oracle_exponent_f64(double v);
int oracle_exponent_f32(float v);
/* Quantise + zfp + shuffle + bit planes of one block (4^ndims doubles).
   Same outputs as the harness's ref_block_encode. Returns the number of coded planes. */
int oracle_block_encode(const double* vals, int ndims, int is_f32, double tol, int bpc,
                        int* emax, uint64_t* ucoeffs, int* plane_bp, int* plane_nin,
                        int* plane_bits, uint64_t* plane_words);
int oracle_block_decode(int ndims, int emax, int nplanes, const int* plane_bp,
                        const uint64_t* plane_words, double* out_vals);

/* varbyte(vals[i]) for i < n_var, then unary(vals[i]) (Core/VarInt.h:14,82). */
long long oracle_varint_stream(const uint64_t* vals, int n_var, int n_total, uint8_t* out,
                               long long cap);

uint32_t oracle_encode_morton3(uint32_t x, uint32_t y, uint32_t z);

#ifdef __cplusplus
}
#endif

#endif
