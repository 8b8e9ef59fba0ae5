// Device packer, device side (dpack_device.h): the launches of the key pass and k_pack_write
// between the host stages of dpack_plan.cpp, and the encode path that uses them.
#include "dpack_device.h"

#include "trace.h"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <fcntl.h>
#include <thread>
#include <unistd.h>

namespace idx2g
{

namespace
{

// The segment tables of one plan, on the host and uploaded (kept on the context).
struct dpack_tables
{
  std::shared_ptr<const encode_plan> plan;  // (kept alive: the key is its identity)
  std::vector<std::vector<int>> nexps;
  std::vector<unsigned> bricks_per_chunk;
  dpack_plan P;
  std::vector<int4> subs;
  std::vector<int> seg_sub0;
  dpack_segment* d_segs = nullptr;
  dpack_event* d_evs = nullptr;
  int4* d_subs = nullptr;
  int* d_sub0 = nullptr;
};

} // namespace

int device_pack(device_ctx* ctx, const dataset_format& f, const std::shared_ptr<const encode_plan>& plan,
                const std::vector<device_level_stream>& levels, packed_dataset* out, const image_hook& on_image)
{
  stage_timer tt;
  cudaStream_t st = ctx->stream;
  if (levels.size() > 16 || !plan)
    return InvalidArgument;
  std::vector<std::vector<int>> nexps(levels.size());
  for (size_t l = 0; l < levels.size(); ++l)
    nexps[l] = levels[l].nexps;
  std::vector<unsigned> bpc(f.bricks_per_chunk.begin(), f.bricks_per_chunk.end());
  std::shared_ptr<dpack_tables> T = std::static_pointer_cast<dpack_tables>(ctx->dpack);
  if (!T || T->plan != plan || T->nexps != nexps || T->bricks_per_chunk != bpc)
  {
    ctx->dpack.reset();
    T = std::make_shared<dpack_tables>();
    T->plan = plan;
    T->nexps = nexps;
    T->bricks_per_chunk = bpc;
    int e = dpack_make_plan(f, *plan, nexps, &T->P);
    if (e)
      return e;
    // sub-ranges of kPackSub events per segment
    const int ns = (int)T->P.segs.size();
    T->seg_sub0.resize((size_t)ns);
    for (int si = 0; si < ns; ++si)
    {
      T->seg_sub0[(size_t)si] = (int)T->subs.size();
      int q = 0;
      for (int i = T->P.segs[(size_t)si].ev0; i < T->P.segs[(size_t)si].ev1; i += kPackSub, ++q)
        T->subs.push_back(make_int4(si, i, std::min(i + kPackSub, T->P.segs[(size_t)si].ev1), q));
    }
    T->d_segs = (dpack_segment*)ctx->ws("dpack.segs", sizeof(dpack_segment) * (size_t)ns);
    T->d_evs = (dpack_event*)ctx->ws("dpack.evs", sizeof(dpack_event) * T->P.evs.size());
    T->d_subs = (int4*)ctx->ws("dpack.subs", sizeof(int4) * T->subs.size());
    T->d_sub0 = (int*)ctx->ws("dpack.sub0", 4 * (size_t)ns);
    if (!T->d_segs || !T->d_evs || !T->d_subs || !T->d_sub0)
      return OutOfMemory;
    cudaMemcpyAsync(T->d_segs, T->P.segs.data(), sizeof(dpack_segment) * (size_t)ns, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(T->d_evs, T->P.evs.data(), sizeof(dpack_event) * T->P.evs.size(), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(T->d_subs, T->subs.data(), sizeof(int4) * T->subs.size(), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(T->d_sub0, T->seg_sub0.data(), 4 * (size_t)ns, cudaMemcpyHostToDevice, st);
    ctx->dpack = T;
  }
  const dpack_plan& P = T->P;
  const int nseg = (int)P.segs.size();
  dpack_segment* d_segs = T->d_segs;
  dpack_event* d_evs = T->d_evs;
  int* d_kmin = (int*)ctx->ws("dpack.kmin", 4 * (size_t)nseg);
  dpack_key* d_keys = (dpack_key*)ctx->ws("dpack.keys", sizeof(dpack_key) * (size_t)nseg * kSegKeys);
  unsigned long long* d_coff = (unsigned long long*)ctx->ws("dpack.coff", 8 * (size_t)nseg * kSegKeys);
  uint8_t* d_exps = (uint8_t*)ctx->ws("dpack.exps", (size_t)P.exp_total + 16);
  int* d_err = (int*)ctx->ws("dpack.err", 16);
  if (!d_kmin || !d_keys || !d_coff || !d_exps || !d_err)
    return OutOfMemory;
  cudaMemsetAsync(d_err, 0, 16, st);
  const size_t nev = P.evs.size();
  const unsigned long long kb_cap = (unsigned long long)nev * kKeyWindow;
  unsigned long long* d_evreg = (unsigned long long*)ctx->ws("dpack.evreg", 8 * nev);
  int* d_evkmin = (int*)ctx->ws("dpack.evkmin", 4 * nev);
  int* d_evnkeys = (int*)ctx->ws("dpack.evnkeys", 4 * nev);
  unsigned long long* d_evkb = (unsigned long long*)ctx->ws("dpack.evkb", 8 * nev);
  uint32_t* d_kb = (uint32_t*)ctx->ws("dpack.kb", 4 * (size_t)kb_cap);
  unsigned long long* d_cursor = (unsigned long long*)ctx->ws("dpack.cursor", 16);
  int* d_kmax = (int*)ctx->ws("dpack.kmax", 4 * (size_t)nseg);
  dpack_acc* d_acc = (dpack_acc*)ctx->ws("dpack.acc", sizeof(dpack_acc) * (size_t)nseg * kSegKeys);
  dpack_sub* d_subacc = (dpack_sub*)ctx->ws("dpack.subacc", sizeof(dpack_sub) * T->subs.size() * kSegKeys);
  if (!d_evreg || !d_evkmin || !d_evnkeys || !d_evkb || !d_kb || !d_cursor || !d_kmax || !d_acc || !d_subacc)
    return OutOfMemory;
  cudaMemsetAsync(d_cursor, 0, 16, st);
  int e = NoError;
  dpack_args a;
  memset(&a, 0, sizeof a);
  a.segs = d_segs;
  a.nseg = nseg;
  a.evs = d_evs;
  a.nev = (int)nev;
  a.ev_region = d_evreg;
  a.ev_kmin = d_evkmin;
  a.ev_nkeys = d_evnkeys;
  a.ev_kb = d_evkb;
  a.kb = d_kb;
  a.kb_cap = kb_cap;
  a.cursor = d_cursor;
  a.seg_kmax = d_kmax;
  a.acc = d_acc;
  a.subs = T->d_subs;
  a.nsub = (int)T->subs.size();
  a.seg_sub0 = T->d_sub0;
  a.sub_acc = d_subacc;
  for (size_t l = 0; l < levels.size(); ++l)
  {
    a.streams[l] = levels[l].stream;
    a.offsets[l] = levels[l].offset;
  }
  a.etol = exponent_f64(f.tolerance);
  a.end_bp = f.type == dtype::float32 ? 32 : 64;
  a.bpc = f.bit_planes_per_chunk;
  a.exp_bytes = P.exp_bytes;
  a.seg_kmin = d_kmin;
  a.keys = d_keys;
  a.chunk_off = d_coff;
  a.exps = d_exps;
  a.error = d_err;
  // the key pass (a warp per event, a CTA per sub-range for the totals, a CTA per segment for
  // the ranks); k_pack_write: a CTA per sub-range
  const int grid = nseg < 4 * ctx->num_sms ? nseg : 4 * ctx->num_sms;
  const int wgrid = nseg < 2048 ? nseg : 2048;
  dpack_launch_keys(a, grid, st);
  ctx->launches += 4;
  std::vector<dpack_key> keys((size_t)nseg * kSegKeys);
  std::vector<int> kmin((size_t)nseg);
  int err = 0;
  cudaMemcpyAsync(keys.data(), d_keys, sizeof(dpack_key) * keys.size(), cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(kmin.data(), d_kmin, 4 * (size_t)nseg, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(&err, d_err, 4, cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess)
    return CudaError;
  if (err)
    return kDpackNotApplicable;
  tt.lap("dpack.keys");
  out->files.clear();
  out->stats = pack_stats();
  dpack_layout L;
  e = dpack_make_layout(f, P, keys, kmin, &L, out);
  if (e)
    return e;
  tt.lap("dpack.layout");
  const size_t img_words = (size_t)((L.total + 3) / 4) + 1;
  uint32_t* d_img = (uint32_t*)ctx->ws("dpack.image", img_words * 4);
  uint8_t* h_img = (uint8_t*)ctx->pinned("dpack.himage", (size_t)L.total + 16);
  uint8_t* h_exps = (uint8_t*)ctx->pinned("dpack.hexps", (size_t)P.exp_total + 16);
  if (!d_img || !h_img || !h_exps)
    return OutOfMemory;
  cudaMemcpyAsync(d_coff, L.chunk_off.data(), 8 * L.chunk_off.size(), cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(d_img, 0, img_words * 4, st);
  a.image = d_img;
  dpack_launch_write(a, wgrid, st);
  ctx->launches += 1;
  // the raw exponents first: their compression (and the file tails) run on the host while
  // the image comes back
  if (P.exp_total)
    cudaMemcpyAsync(h_exps, d_exps, (size_t)P.exp_total, cudaMemcpyDeviceToHost, st);
  cudaEvent_t ex = ctx->ev(0);
  if (!ex || cudaEventRecord(ex, st) != cudaSuccess)
    return CudaError;
  // the image in pieces, each with an event: the file writer starts on the first pieces
  // while the later ones are still on their way
  constexpr unsigned long long kCopyPiece = 32ull << 20;
  const size_t npiece = (size_t)((L.total + kCopyPiece - 1) / kCopyPiece);
  std::vector<cudaEvent_t> pev(npiece);
  for (size_t i = 0; i < npiece; ++i)
  {
    const unsigned long long o = (unsigned long long)i * kCopyPiece;
    const unsigned long long n = L.total - o < kCopyPiece ? L.total - o : kCopyPiece;
    cudaMemcpyAsync(h_img + o, (const uint8_t*)d_img + o, (size_t)n, cudaMemcpyDeviceToHost, st);
    pev[i] = ctx->ev(1 + i);
    if (!pev[i] || cudaEventRecord(pev[i], st) != cudaSuccess)
      return CudaError;
  }
  const uint8_t* img = h_img;
  const unsigned long long total = L.total;
  out->ready = [pev, img, total](const uint8_t* p, size_t n) {
    if (p < img || p >= img + total || n == 0)
      return;
    const size_t i0 = (size_t)((unsigned long long)(p - img) / kCopyPiece);
    const size_t i1 = (size_t)(((unsigned long long)(p - img) + n - 1) / kCopyPiece);
    for (size_t i = i0; i <= i1 && i < pev.size(); ++i)
      cudaEventSynchronize(pev[i]);
  };
  out->image = h_img;
  if (on_image)
    on_image(L, h_img, out->ready);  // e.g. the chunk sections written while the rest is made
  if (cudaEventSynchronize(ex) != cudaSuccess)
    return CudaError;
  tt.lap("dpack.write");
  e = dpack_finish(f, P, L, h_img, h_exps, out);
  tt.lap("dpack.finish");
  return e;
}

int encode_dataset_dpack(device_ctx* ctx, dataset_format* f, params* p, gpu_coder* coder, encode_timing* timing,
                         const std::shared_ptr<const encode_plan>& plan_sp,
                         const std::vector<unsigned long long>* prealloc)
{
  const encode_plan& plan = *plan_sp;
  auto now = [] { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); };
  const double t0 = now();
  std::thread pre;
  if (prealloc)
    pre = preallocate_files(*f, plan, *prealloc);
  struct joiner
  {
    std::thread& t;
    ~joiner()
    {
      if (t.joinable())
        t.join();
    }
  } join_pre{ pre };
  coder->set_keep_device(true);
  std::vector<level_output> outs;
  int e = encode_levels(f, coder, &outs, plan);
  if (e)
    return e;
  const double t1 = now();
  std::vector<device_level_stream> lv(outs.size());
  for (size_t l = 0; l < outs.size(); ++l)
  {
    coder->device_level((int)l, &lv[l].stream, &lv[l].offset);
    lv[l].nsb = outs[l].nsb;
    lv[l].nexps = outs[l].nexps;
  }
  // the chunk sections (most of every file) are written, on a thread, as their pieces arrive
  // from the device, while the host compresses the exponent chunks and builds the tails
  std::map<std::string, unsigned long long> sec_bytes;
  std::map<std::string, file_buffer> sec_files;
  int sec_err = NoError;
  std::thread sections;
  struct section_joiner  // (declared after what the thread uses: joined before those go)
  {
    std::thread& t;
    ~section_joiner()
    {
      if (t.joinable())
        t.join();
    }
  } join_sections{ sections };
  const image_hook on_image = [&](const dpack_layout& L, const uint8_t* img, const ready_fn& ready) {
    for (const auto& kv : L.file_span)
    {
      sec_bytes[kv.first] = kv.second.second;
      file_buffer& fb = sec_files[kv.first];
      constexpr unsigned long long kPiece = 16ull << 20;
      for (unsigned long long o = 0; o < kv.second.second; o += kPiece)
        fb.append_ref(img + kv.second.first + o,
                      (size_t)(kv.second.second - o < kPiece ? kv.second.second - o : kPiece));
    }
    sections = std::thread([&, ready]() {
      stage_timer ts;
      if (pre.joinable())
        pre.join();
      std::vector<std::pair<std::string, const file_buffer*>> wl;
      for (auto& kv : sec_files)
        wl.push_back({ kv.first, &kv.second });
      sec_err = write_files(wl, &ready);
      ts.lap("write.sections (thread)");
    });
  };
  packed_dataset pd;
  e = device_pack(ctx, *f, plan_sp, lv, &pd, on_image);
  if (e && e != kDpackNotApplicable)
    cudaStreamSynchronize(ctx->stream);  // (no copy left running into the pinned image)
  if (e == kDpackNotApplicable)
  {
    // a segment with more keys than the kernels' window: the regions to the host packer
    e = NoError;
    for (size_t l = 0; l < outs.size() && !e; ++l)
      e = coder->copy_level_out((int)l, &outs[l]);
    if (e)
      return e;
    e = pack_dataset(f, p, plan, outs, nullptr, true, timing, &pre);
    if (timing)
      timing->device_s = t1 - t0;
    return e;
  }
  if (e)
    return e;
  if (timing)
    note_level_files(*f, plan, pd.files, timing);
  const double t2 = now();
  stage_timer tw;
  if (sections.joinable())
    sections.join();
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess)
    return CudaError;
  if (sec_err)
    return sec_err;
  tw.lap("write.sections_wait");
  // the rest of every file after its chunk section, and the metadata file
  const std::string meta = meta_text(*f, *p) + pack_stats_text(pd.stats);
  e = write_file(p->out_dir + "/" + p->name + "/" + p->field + ".idx2", std::vector<uint8_t>(meta.begin(), meta.end()));
  unsigned long long total = meta.size();
  for (auto& kv : pd.files)
  {
    if (e)
      break;
    const file_buffer& fb = kv.second;
    total += fb.nbytes;
    const unsigned long long skip = sec_bytes.count(kv.first) ? sec_bytes[kv.first] : 0;
    if (!skip && make_dirs_for(kv.first) != NoError)
    {
      e = CannotCreateDirectory;
      break;
    }
    const int fd = open(kv.first.c_str(), O_RDWR | O_CREAT | (skip ? 0 : O_TRUNC), 0644);
    if (fd < 0)
    {
      e = FileCreateFailed;
      break;
    }
    unsigned long long at = 0;
    fb.for_each_segment([&](const segment& sg) {
      if (e)
        return;
      const unsigned long long a0 = at, a1 = at + sg.n;
      at = a1;
      if (a1 <= skip)
        return;  // in the chunk section, written already
      const unsigned long long from = a0 < skip ? skip - a0 : 0;
      size_t done = (size_t)from;
      while (done < sg.n)
      {
        const ssize_t w = pwrite(fd, sg.p + done, sg.n - done, (off_t)(a0 + done));
        if (w <= 0)
        {
          e = FileWriteFailed;
          return;
        }
        done += (size_t)w;
      }
    });
    if (!e && ftruncate(fd, (off_t)fb.nbytes) != 0)
      e = FileWriteFailed;
    if (close(fd) != 0 && !e)
      e = FileWriteFailed;
  }
  const double t3 = now();
  tw.lap("write.tails");
  if (timing)
  {
    timing->device_s = t1 - t0;
    timing->pack_s = t2 - t1;
    timing->write_s = t3 - t2;
    timing->file_bytes = total;
    timing->nfiles = (int)pd.files.size() + 1;
  }
  return e;
}

} // namespace idx2g
