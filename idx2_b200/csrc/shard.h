// One encode split over several processes (one GPU each), with no exchange of coded data.
//
// The reference encodes depth first (Core/idx2Encode.cpp:276-340): every brick of the
// coarsest level owns an independent subtree, the level-0 bricks under it and every brick
// between. A shard takes a contiguous run of the coarsest level's bricks (in encode order)
// and codes exactly their subtrees. The chunk and file layout depends on the coded streams
// only through their sizes, so the shards exchange the headers of their (brick, subband)
// regions (channel keys, block exponents, channel byte sizes: a few hundred bytes per
// brick and subband); every shard then replays the reference's packing over all headers
// (the same layout on every shard) and writes into the shared files the bytes it owns: its
// bricks' channel streams. Shard 0 also writes every byte made while packing (chunk headers,
// the zstd exponent chunks, tables and tails) and the metadata file. Files are written with
// positional writes at offsets every shard computes alike, so the writes do not overlap.
#pragma once

#include "encoder.h"

#include <vector>

namespace idx2g
{

struct shard_plan
{
  int nshards = 1, shard = 0;
  std::vector<std::vector<int>> owner;        // [level][brick] -> shard
  std::vector<std::vector<int>> local_index;  // [level][brick] -> index in `local`, -1 if another shard's
  encode_plan local;                          // this shard's bricks and events, in encode order
  extent region;                              // bounding box (samples) of this shard's level-0 bricks
};

// Split the plan of format f into nshards runs of coarsest bricks (sizes differing by at most
// one) and describe shard `shard`.
int make_shard_plan(const dataset_format& f, const encode_plan& plan, int nshards, int shard, shard_plan* sp);

// The exchange payload of a shard: the headers of its (brick, subband) regions in the global
// event order (outs are the shard's level outputs, indexed by the local plan).
int shard_headers(const dataset_format& f, const encode_plan& plan, const shard_plan& sp,
                  const std::vector<level_output>& outs, std::vector<uint8_t>* blob);

// Pack with the headers of every shard (blobs[s], sizes[s] for shard s) and write this shard's
// part of every data file; shard 0 also writes the metadata file. f's value range must be the
// whole field's (the caller reduces it over the shards).
int pack_shard(const dataset_format* f, const params* p, const encode_plan& plan, const shard_plan& sp,
               const std::vector<level_output>& outs, const std::vector<const uint8_t*>& blobs,
               const std::vector<size_t>& sizes, encode_timing* timing);

} // namespace idx2g
