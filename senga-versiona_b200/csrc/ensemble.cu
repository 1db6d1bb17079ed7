// Batched ensembles and the serving loop.
//
// An Ensemble holds many independent periodic boxes of uneven sizes that
// share one mechanism. All their fields live in one HBM arena (first-fit
// allocator over a single device allocation); each box has a descriptor
// (geometry, field pointers, the five RK coefficient triples of its own dt).
// One RK substage of the whole ensemble runs in one of two forms:
//   * persistent: one launch per substage (per table of up to 64 boxes) of
//     the kernel of persist.cu, whose resident CTAs take the thermochemistry
//     chunks and the flow, species and species+RK tiles of every box from one
//     phase-major work list, each phase of a box starting when the box's
//     previous phase has completed;
//   * four launches: the pointwise thermochemistry over (box, 256-point
//     chunk) items and the three stencil kernels over (box, tile) items.
// The RK step (five substages) is captured once as a CUDA graph and
// replayed. The autotuner times one RK step of the live ensemble for each
// candidate (the persistent kernel at 1..k resident CTAs per SM; the four
// launches at several thermochemistry grid sizes) and keeps the fastest;
// SENGA_BATCH=persist or =launches restricts it to one form.
//
// The serving loop (senga_server_*) keeps an Ensemble whose membership
// changes between RK steps: requests are admitted as soon as the arena has
// room for their fields (admission by HBM footprint), every active request
// advances one RK step per tick together with all the others, and finished
// requests are copied back to the host and their memory released. A tick
// never waits for the device except to keep at most two steps queued: every
// copy goes through page-locked staging (so it queues behind the kernels
// instead of waiting for them), work lists are uploaded in stream order, the
// steps are launched kernel by kernel (membership changes most ticks), and a
// result is handed to the host by an event callback once its download has
// completed.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "senga_gpu.h"
#include "senga_internal.h"

namespace senga {
namespace {

#define CKE(call)                                                                             \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess)                                                                    \
      throw Error(e_ == cudaErrorMemoryAllocation ? SENGA_ERR_NOMEM : SENGA_ERR_CUDA,         \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                        \
  } while (0)

const double kA[5] = {970286171893.0 / 4311952581923.0, 6584761158862.0 / 12103376702013.0,
                      2251764453980.0 / 15575788980749.0, 26877169314380.0 / 34165994151039.0, 0.0};
const double kB[5] = {1153189308089.0 / 22510343858157.0, 1772645290293.0 / 4653164025191.0,
                      -1672844663538.0 / 4480602732383.0, 2114624349019.0 / 3568978502595.0,
                      5198255086312.0 / 14908931495163.0};
const double kBh[5] = {1016888040809.0 / 7410784769900.0, 11231460423587.0 / 58533540763752.0,
                       -1563879915014.0 / 6823010717585.0, 606302364029.0 / 971179775848.0,
                       1097981568119.0 / 3980877426909.0};

// First-fit allocator over one device allocation (256-byte granules).
class Arena {
 public:
  void init(size_t bytes) {
    cap_ = (bytes + 255) / 256;
    CKE(cudaMalloc(&base_, cap_ * 256));
    free_.clear();
    free_[0] = cap_;
  }
  void release_all() {
    if (base_) cudaFree(base_);
    base_ = nullptr;
  }
  // returns nullptr when no hole is large enough
  void* take(size_t bytes) {
    const size_t g = (bytes + 255) / 256;
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= g) {
        const size_t off = it->first, len = it->second;
        free_.erase(it);
        if (len > g) free_[off + g] = len - g;
        used_[off] = g;
        return static_cast<char*>(base_) + off * 256;
      }
    }
    return nullptr;
  }
  void give(void* p) {
    const size_t off = (static_cast<char*>(p) - static_cast<char*>(base_)) / 256;
    auto u = used_.find(off);
    if (u == used_.end()) return;
    size_t len = u->second;
    used_.erase(u);
    size_t start = off;
    auto nx = free_.lower_bound(off);
    if (nx != free_.end() && nx->first == off + len) {
      len += nx->second;
      free_.erase(nx);
    }
    auto pv = free_.lower_bound(off);
    if (pv != free_.begin()) {
      --pv;
      if (pv->first + pv->second == off) {
        start = pv->first;
        len += pv->second;
        free_.erase(pv);
      }
    }
    free_[start] = len;
  }
  size_t free_bytes() const {
    size_t s = 0;
    for (auto& kv : free_) s += kv.second;
    return s * 256;
  }
  size_t capacity() const { return cap_ * 256; }

 private:
  void* base_ = nullptr;
  size_t cap_ = 0;
  std::map<size_t, size_t> free_, used_;
};

size_t box_bytes(const senga_config& c, int nspec) {
  const int64_t n = (int64_t)c.nx * c.ny * c.nz;
  const int nc = 5 + nspec;
  const int64_t dbl = (int64_t)(3 * nc + 4 * nspec + 15) * n + (n + 1) / 2 + 64;
  return (size_t)dbl * sizeof(double);
}

void check_box(const senga_config& c) {
  const int n3[3] = {c.nx, c.ny, c.nz};
  for (int d = 0; d < 3; ++d) {
    if (n3[d] < 11) throw Error(SENGA_ERR_ARG, "ensemble boxes need at least 11 points per direction");
    if (c.nend[2 * d] != SENGA_NPERI || c.nend[2 * d + 1] != SENGA_NPERI)
      throw Error(SENGA_ERR_UNSUPPORTED, "ensemble boxes must be periodic");
  }
  if (c.tstep <= 0.0) throw Error(SENGA_ERR_ARG, "tstep must be positive");
}

// Page-locked staging for the serving loop's copies: a FIFO ring of chunks,
// each released once the copy through it has completed (its event) and, for
// a download, once the host has taken the data out. Copies from page-locked
// memory run on the stream without waiting for the kernels queued before
// them, so admitting or retiring a request never stalls the device.
class PinnedRing {
 public:
  struct Chunk {
    size_t off = 0, len = 0;
    cudaEvent_t ev = nullptr;
    std::function<void(const char*)> done;  // run on the host once the copy has completed
  };
  void init(size_t bytes) {
    cap_ = bytes;
    CKE(cudaMallocHost(&base_, cap_));
  }
  void release_all() {
    for (Chunk& c : q_)
      if (c.ev) cudaEventDestroy(c.ev);
    q_.clear();
    if (base_) cudaFreeHost(base_);
    base_ = nullptr;
  }
  // a chunk of `bytes` (rounded up to 256); waits for the oldest copies when
  // the ring is full
  Chunk* take(size_t bytes) {
    bytes = (bytes + 255) / 256 * 256;
    if (bytes > cap_) throw Error(SENGA_ERR_NOMEM, "pinned staging smaller than one request");
    for (;;) {
      reclaim();
      size_t off = 0;
      if (!q_.empty()) {
        const size_t tail = q_.back().off + q_.back().len, head = q_.front().off;
        if (tail >= head) {  // free: [tail, cap) and [0, head)
          if (cap_ - tail >= bytes) off = tail;
          else if (head >= bytes) off = 0;
          else off = SIZE_MAX;
        } else {  // free: [tail, head)
          off = head - tail >= bytes ? tail : SIZE_MAX;
        }
      }
      if (off != SIZE_MAX) {
        Chunk c;
        c.off = off;
        c.len = bytes;
        CKE(cudaEventCreateWithFlags(&c.ev, cudaEventDisableTiming));
        q_.push_back(c);
        return &q_.back();
      }
      // full: wait for the oldest chunk's copy
      CKE(cudaEventSynchronize(q_.front().ev));
    }
  }
  // wait for the oldest copy in flight (false when none)
  bool wait_oldest() {
    if (q_.empty()) return false;
    CKE(cudaEventSynchronize(q_.front().ev));
    reclaim();
    return true;
  }
  char* ptr(const Chunk* c) const { return static_cast<char*>(base_) + c->off; }
  // retire the completed chunks from the head (copies on one stream complete
  // in order), running their host callbacks
  void reclaim() {
    while (!q_.empty() && cudaEventQuery(q_.front().ev) == cudaSuccess) {
      Chunk c = q_.front();
      q_.pop_front();
      if (c.done) c.done(static_cast<const char*>(base_) + c.off);
      cudaEventDestroy(c.ev);
    }
  }

 private:
  void* base_ = nullptr;
  size_t cap_ = 0;
  std::deque<Chunk> q_;
};

struct Member {
  int id = -1;
  senga_config cfg{};
  BoxDesc desc{};
  void* block = nullptr;
  int steps_left = 0;   // serving: RK steps still to run
  int steps_done = 0;
  double t_submit = 0.0, t_admit = 0.0, t_done = 0.0;
  // serving: host copies of the initial state until admission, result after
  std::vector<double> h_fields, h_t;
  std::vector<int32_t> h_itn;
  bool finishing = false;  // serving: last step queued, result not yet on the host
};

class Ensemble {
 public:
  senga_chem chem{};
  senga_diff diff{};
  int nspec = 0, nc = 0, mech = 0, device = 0;
  cudaStream_t stream = nullptr;
  senga_chem* d_chem = nullptr;
  senga_diff* d_diff = nullptr;
  unsigned int* d_status = nullptr;
  Arena arena;
  std::vector<Member*> active;
  int grid_stencil = 0, grid_thermo = 0;
  bool persist = false;  // one persistent launch per substage
  int grid_persist = 0;

  void init(const senga_chem& c, const senga_diff* d, int dev, size_t arena_bytes) {
    chem = c;
    if (d) diff = *d;
    else std::memset(&diff, 0, sizeof(diff));
    nspec = c.nspec;
    // the batched thermochemistry kernels are built for up to 9 species
    // (one ITNDEX word); the larger mechanisms run as single contexts
    if (nspec < 1 || nspec > 9)
      throw Error(SENGA_ERR_UNSUPPORTED, "batched ensembles and the serving loop take mechanisms of at most 9 species");
    nc = 5 + nspec;
    device = dev;
    mech = select_mech(chem, diff);
    CKE(cudaSetDevice(dev));
    CKE(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    CKE(cudaMalloc(&d_chem, sizeof(senga_chem)));
    CKE(cudaMalloc(&d_diff, sizeof(senga_diff)));
    CKE(cudaMemcpy(d_chem, &chem, sizeof(senga_chem), cudaMemcpyHostToDevice));
    CKE(cudaMemcpy(d_diff, &diff, sizeof(senga_diff), cudaMemcpyHostToDevice));
    CKE(cudaMalloc(&d_status, sizeof(unsigned int)));
    CKE(cudaMemset(d_status, 0, sizeof(unsigned int)));
    arena.init(arena_bytes);
    int sms = 0;
    CKE(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    sms_ = sms;
    grid_thermo = 4 * sms;
    persist_occ_ = std::max(1, persist_ctas_per_sm(mech, nspec, diff.flmavt));
    grid_persist = persist_occ_ * sms;
    const char* e = std::getenv("SENGA_BATCH");
    form_ = e ? std::string(e) : std::string();
    persist = form_ == "persist";
  }
  void destroy() {
    drop_graph();
    if (stream) cudaStreamSynchronize(stream);
    cudaFree(d_items_);
    cudaFree(d_chunks_);
    cudaFree(d_pitems_);
    cudaFree(d_need_);
    cudaFree(d_ctr_);
    cudaFree(d_chem);
    cudaFree(d_diff);
    cudaFree(d_status);
    arena.release_all();
    if (stream) cudaStreamDestroy(stream);
  }

  // places a member's fields in the arena; false when it does not fit
  bool place(Member& m) {
    const size_t bytes = box_bytes(m.cfg, nspec);
    void* blk = arena.take(bytes);
    if (!blk) return false;
    m.block = blk;
    BoxDesc& b = m.desc;
    std::memset(&b, 0, sizeof(b));
    const senga_config& c = m.cfg;
    b.g.nx = c.nx;
    b.g.ny = c.ny;
    b.g.nz = c.nz;
    b.g.n = (int64_t)c.nx * c.ny * c.nz;
    const int n3[3] = {c.nx, c.ny, c.nz};
    const double len[3] = {c.xgdlen, c.ygdlen, c.zgdlen};
    for (int d = 0; d < 3; ++d) {
      b.g.per[d] = 1;
      const double delta = len[d] / (double)(float)(n3[d] - 1);
      b.g.ovd[d] = 1.0 / delta;
      b.g.ovd2[d] = b.g.ovd[d] * b.g.ovd[d];
    }
    for (int i = 0; i < 5; ++i) {
      b.rk[i].lhs = kB[i] * c.tstep;
      b.rk[i].rhs = kA[i] * c.tstep;
      b.rk[i].err = (kB[i] - kBh[i]) * c.tstep;
      b.rk[i].last = i == 4 ? 1 : 0;
    }
    b.nspec = nspec;
    const int64_t n = b.g.n;
    double* p = static_cast<double*>(blk);
    auto take = [&](int64_t k) {
      double* r = p;
      p += k * n;
      return r;
    };
    Fields& f = b.f;
    f.run = take(nc);
    f.uin = take(nc);
    f.uout = f.uin;
    f.err = nullptr;
    f.t = take(1);
    f.p = take(1);
    f.lam = take(1);
    f.lcp = take(1);
    f.mu = take(1);
    f.rd = take(nspec);
    f.h = take(nspec);
    f.hmix = take(1);
    f.wdot = take(nspec);
    f.vel = take(3);
    f.e = take(1);
    f.y = take(nspec);
    f.rhs = take(nc);
    f.divm = take(1);
    f.vc = take(3);
    f.vtmp = take(1);
    f.itn = reinterpret_cast<int32_t*>(p);
    f.status = d_status;
    return true;
  }
  void unplace(Member& m) {
    if (m.block) arena.give(m.block);
    m.block = nullptr;
  }
  void upload(Member& m, const double* fields, const double* t, const int32_t* itn) {
    const int64_t n = m.desc.g.n;
    const size_t bytes = (size_t)nc * n * sizeof(double);
    CKE(cudaMemcpyAsync(m.desc.f.run, fields, bytes, cudaMemcpyHostToDevice, stream));
    CKE(cudaMemcpyAsync(m.desc.f.uin, m.desc.f.run, bytes, cudaMemcpyDeviceToDevice, stream));
    CKE(cudaMemcpyAsync(m.desc.f.t, t, n * sizeof(double), cudaMemcpyHostToDevice, stream));
    CKE(cudaMemcpyAsync(m.desc.f.itn, itn, n * sizeof(int32_t), cudaMemcpyHostToDevice, stream));
  }
  void download(Member& m, double* fields, double* t, int32_t* itn) {
    const int64_t n = m.desc.g.n;
    CKE(cudaMemcpyAsync(fields, m.desc.f.run, (size_t)nc * n * sizeof(double), cudaMemcpyDeviceToHost, stream));
    if (t) CKE(cudaMemcpyAsync(t, m.desc.f.t, n * sizeof(double), cudaMemcpyDeviceToHost, stream));
    if (itn) CKE(cudaMemcpyAsync(itn, m.desc.f.itn, n * sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
  }

  // rebuild descriptors and work lists of the active members: boxes go into
  // tables of kTableBoxes, each with its contiguous run of tiles and chunks
  void rebuild(PinnedRing* ring = nullptr) {
    drop_graph();
    groups_.clear();
    grid_stencil = 0;
    std::vector<WorkItem> items, chunks;
    int tx, ty, tz;
    tile_shape(&tx, &ty, &tz);
    const int tb = thermo_block();
    for (size_t k = 0; k < active.size(); ++k) {
      const int local = (int)(k % kTableBoxes);
      if (local == 0) {
        groups_.emplace_back();
        Group& gr = groups_.back();
        gr.table.reset(new BoxTable());
        std::memset(gr.table.get(), 0, sizeof(BoxTable));
        gr.item0 = (int)items.size();
        gr.chunk0 = (int)chunks.size();
      }
      Group& gr = groups_.back();
      const BoxDesc& b = active[k]->desc;
      gr.table->d[local] = b;
      const int bx = (b.g.nx + tx - 1) / tx, by = (b.g.ny + ty - 1) / ty, bz = (b.g.nz + tz - 1) / tz;
      for (int z = 0; z < bz; ++z)
        for (int y = 0; y < by; ++y)
          for (int x = 0; x < bx; ++x) items.push_back(WorkItem{local, x * tx, y * ty, z * tz});
      const int64_t nch = (b.g.n + tb - 1) / tb;
      for (int64_t c = 0; c < nch; ++c) chunks.push_back(WorkItem{local, (int)c, 0, 0});
      gr.nitems = (int)items.size() - gr.item0;
      grid_stencil = (int)items.size();
      gr.nchunks = (int)chunks.size() - gr.chunk0;
    }
    // persistent form: per table, the chunks then three copies of the tiles
    // (flow, species, species+RK), and the items of every (box, phase)
    std::vector<WorkItem> pitems;
    std::vector<int> need((size_t)groups_.size() * 4 * kTableBoxes, 0);
    for (size_t gi = 0; gi < groups_.size(); ++gi) {
      Group& gr = groups_[gi];
      gr.pitem0 = (int)pitems.size();
      gr.poff[0] = 0;
      for (int c = 0; c < gr.nchunks; ++c) pitems.push_back(chunks[gr.chunk0 + c]);
      for (int ph = 1; ph < 4; ++ph) {
        gr.poff[ph] = (int)pitems.size() - gr.pitem0;
        for (int k = 0; k < gr.nitems; ++k) pitems.push_back(items[gr.item0 + k]);
      }
      gr.poff[4] = (int)pitems.size() - gr.pitem0;
      int* nd = need.data() + gi * 4 * kTableBoxes;
      for (int c = 0; c < gr.nchunks; ++c) ++nd[4 * chunks[gr.chunk0 + c].box];
      for (int k = 0; k < gr.nitems; ++k)
        for (int ph = 1; ph < 4; ++ph) ++nd[4 * items[gr.item0 + k].box + ph];
    }
    std::vector<int> zeros((size_t)groups_.size() * kPersistCounters, 0);
    if (ring) {  // serving: through the page-locked ring, stream-ordered, no wait
      staged_upload(*ring, items, &d_items_, &cap_items_);
      staged_upload(*ring, chunks, &d_chunks_, &cap_chunks_);
      staged_upload(*ring, pitems, &d_pitems_, &cap_pitems_);
      staged_upload(*ring, need, &d_need_, &cap_need_);
      staged_upload(*ring, zeros, &d_ctr_, &cap_ctr_);
      return;
    }
    upload_vec(items, &d_items_, &cap_items_);
    upload_vec(chunks, &d_chunks_, &cap_chunks_);
    upload_vec(pitems, &d_pitems_, &cap_pitems_);
    upload_vec(need, &d_need_, &cap_need_);
    upload_vec(zeros, &d_ctr_, &cap_ctr_);
    CKE(cudaStreamSynchronize(stream));
  }
  void substage(int irk) {
    if (active.empty()) return;
    if (persist) {
      for (size_t gi = 0; gi < groups_.size(); ++gi) {
        const Group& gr = groups_[gi];
        PersistArgs a{};
        a.items = d_pitems_ + gr.pitem0;
        for (int k = 0; k < 5; ++k) a.off[k] = gr.poff[k];
        a.need = d_need_ + gi * 4 * kTableBoxes;
        a.ctr = d_ctr_ + gi * kPersistCounters;
        a.irk = irk - 1;
        launch_batch_persist(*gr.table, a, grid_persist, mech, d_chem, d_diff, nspec, diff.flmavt, stream);
      }
      return;
    }
    for (const Group& gr : groups_)
      launch_batch_thermo(*gr.table, d_chunks_ + gr.chunk0, gr.nchunks, std::min(grid_thermo, gr.nchunks), mech,
                          d_chem, d_diff, nspec, diff.flmavt, stream);
    for (int phase = 0; phase < 3; ++phase)
      for (const Group& gr : groups_)
        launch_batch_stencil(*gr.table, d_items_ + gr.item0, gr.nitems, irk - 1, phase, stream);
  }
  // one RK step launched kernel by kernel (the serving loop: its membership
  // changes most ticks, so a graph would be captured anew each time)
  void step_direct() {
    for (int irk = 1; irk <= 5; ++irk) substage(irk);
    CKE(cudaGetLastError());
  }
  void step_graph(int nsteps) {
    if (active.empty()) return;
    if (!graph_) {
      cudaGraph_t g;
      CKE(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
      for (int irk = 1; irk <= 5; ++irk) substage(irk);
      CKE(cudaStreamEndCapture(stream, &g));
      CKE(cudaGraphInstantiate(&graph_, g, 0));
      CKE(cudaGraphDestroy(g));
    }
    for (int s = 0; s < nsteps; ++s) CKE(cudaGraphLaunch(graph_, stream));
    CKE(cudaGetLastError());
  }
  // Times one RK step per candidate on the live ensemble (state saved and
  // restored) and keeps the fastest: the persistent kernel at 1..k resident
  // CTAs per SM (k its occupancy), the four launches at 2..32 pointwise CTAs
  // per SM (their stencil kernels launch one CTA per tile).
  void autotune() {
    if (active.empty()) return;
    // save registers, T and ITNDEX of every member
    std::vector<void*> saves;
    for (Member* m : active) {
      const int64_t n = m->desc.g.n;
      const size_t bytes = (size_t)(2 * nc + 1) * n * sizeof(double) + (size_t)n * sizeof(int32_t);
      void* s = nullptr;
      CKE(cudaMalloc(&s, bytes));
      CKE(cudaMemcpyAsync(s, m->desc.f.run, (size_t)(2 * nc) * n * sizeof(double), cudaMemcpyDeviceToDevice, stream));
      CKE(cudaMemcpyAsync(static_cast<char*>(s) + (size_t)(2 * nc) * n * sizeof(double), m->desc.f.t, n * sizeof(double),
                          cudaMemcpyDeviceToDevice, stream));
      CKE(cudaMemcpyAsync(static_cast<char*>(s) + (size_t)(2 * nc + 1) * n * sizeof(double), m->desc.f.itn,
                          n * sizeof(int32_t), cudaMemcpyDeviceToDevice, stream));
      saves.push_back(s);
    }
    cudaEvent_t e0, e1;
    CKE(cudaEventCreate(&e0));
    CKE(cudaEventCreate(&e1));
    struct Cand {
      bool persist;
      int grid;
    };
    std::vector<Cand> cands;
    if (form_ != "launches")
      for (int k = 1; k <= persist_occ_; ++k) cands.push_back(Cand{true, k * sms_});
    if (form_ != "persist")
      for (int t : {2, 4, 8, 16, 32}) cands.push_back(Cand{false, t * sms_});
    float best = 1e30f;
    Cand win = cands.front();
    for (const Cand& cd : cands) {
      persist = cd.persist;
      if (cd.persist) grid_persist = cd.grid;
      else grid_thermo = cd.grid;
      for (int irk = 1; irk <= 5; ++irk) substage(irk);  // warm
      CKE(cudaEventRecord(e0, stream));
      for (int irk = 1; irk <= 5; ++irk) substage(irk);
      CKE(cudaEventRecord(e1, stream));
      CKE(cudaEventSynchronize(e1));
      float ms = 0.f;
      CKE(cudaEventElapsedTime(&ms, e0, e1));
      if (ms < best) {
        best = ms;
        win = cd;
      }
    }
    persist = win.persist;
    if (win.persist) grid_persist = win.grid;
    else grid_thermo = win.grid;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    for (size_t k = 0; k < active.size(); ++k) {
      Member* m = active[k];
      const int64_t n = m->desc.g.n;
      CKE(cudaMemcpyAsync(m->desc.f.run, saves[k], (size_t)(2 * nc) * n * sizeof(double), cudaMemcpyDeviceToDevice, stream));
      CKE(cudaMemcpyAsync(m->desc.f.t, static_cast<char*>(saves[k]) + (size_t)(2 * nc) * n * sizeof(double),
                          n * sizeof(double), cudaMemcpyDeviceToDevice, stream));
      CKE(cudaMemcpyAsync(m->desc.f.itn, static_cast<char*>(saves[k]) + (size_t)(2 * nc + 1) * n * sizeof(double),
                          n * sizeof(int32_t), cudaMemcpyDeviceToDevice, stream));
    }
    CKE(cudaStreamSynchronize(stream));
    for (void* s : saves) cudaFree(s);
    drop_graph();
  }
  void drop_graph() {
    if (graph_) cudaGraphExecDestroy(graph_);
    graph_ = nullptr;
  }

 private:
  // the same through a page-locked chunk; a device array that must grow is
  // reallocated with room to spare (cudaFree waits for the device)
  template <class T>
  void staged_upload(PinnedRing& ring, const std::vector<T>& v, T** d, size_t* cap) {
    if (v.empty()) return;
    if (v.size() > *cap) {
      cudaFree(*d);
      *d = nullptr;
      CKE(cudaMalloc(d, 2 * v.size() * sizeof(T)));
      *cap = 2 * v.size();
    }
    PinnedRing::Chunk* c = ring.take(v.size() * sizeof(T));
    std::memcpy(ring.ptr(c), v.data(), v.size() * sizeof(T));
    CKE(cudaMemcpyAsync(*d, ring.ptr(c), v.size() * sizeof(T), cudaMemcpyHostToDevice, stream));
    CKE(cudaEventRecord(c->ev, stream));
  }
  template <class T>
  void upload_vec(const std::vector<T>& v, T** d, size_t* cap) {
    if (v.empty()) return;
    if (v.size() > *cap) {
      cudaFree(*d);
      *d = nullptr;
      CKE(cudaMalloc(d, v.size() * sizeof(T)));
      *cap = v.size();
    }
    CKE(cudaMemcpyAsync(*d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, stream));
  }
  int sms_ = 148;
  int persist_occ_ = 1;
  std::string form_;  // SENGA_BATCH: "persist", "launches" or empty (both)
  struct Group {
    std::unique_ptr<BoxTable> table;
    int item0 = 0, nitems = 0, chunk0 = 0, nchunks = 0;
    int pitem0 = 0, poff[5] = {};
  };
  std::vector<Group> groups_;
  WorkItem* d_items_ = nullptr;
  WorkItem* d_chunks_ = nullptr;
  WorkItem* d_pitems_ = nullptr;
  int* d_need_ = nullptr;
  int* d_ctr_ = nullptr;
  size_t cap_items_ = 0, cap_chunks_ = 0, cap_pitems_ = 0, cap_need_ = 0, cap_ctr_ = 0;
  cudaGraphExec_t graph_ = nullptr;
};

template <class Fn>
int guard2(Fn&& fn) {
  try {
    fn();
    return SENGA_OK;
  } catch (const Error& e) {
    return fail(e.code, e.what());
  } catch (const std::exception& e) {
    return fail(SENGA_ERR_CUDA, e.what());
  }
}

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

}  // namespace
}  // namespace senga

using namespace senga;

// ============================================================================
struct senga_batch {
  Ensemble ens;
  std::vector<Member> members;
};

extern "C" {

int senga_batch_create(int nbox, const senga_config* cfgs, const senga_chem* chem, const senga_diff* diff, int device,
                       senga_batch** out) {
  if (nbox < 1 || !cfgs || !chem || !out) return fail(SENGA_ERR_ARG, "senga_batch_create: bad argument");
  *out = nullptr;
  senga_batch* b = new senga_batch();
  int rc = guard2([&] {
    size_t total = 0;
    for (int i = 0; i < nbox; ++i) {
      check_box(cfgs[i]);
      total += (box_bytes(cfgs[i], chem->nspec) + 511) / 256 * 256;
    }
    b->ens.init(*chem, diff, device, total);
    b->members.resize(nbox);
    for (int i = 0; i < nbox; ++i) {
      b->members[i].id = i;
      b->members[i].cfg = cfgs[i];
      if (!b->ens.place(b->members[i])) throw Error(SENGA_ERR_NOMEM, "senga_batch_create: arena too small");
      b->ens.active.push_back(&b->members[i]);
    }
    b->ens.rebuild();
  });
  if (rc != SENGA_OK) {
    b->ens.destroy();
    delete b;
    return rc;
  }
  *out = b;
  return SENGA_OK;
}

int senga_batch_destroy(senga_batch* b) {
  if (!b) return SENGA_OK;
  b->ens.destroy();
  delete b;
  return SENGA_OK;
}

int senga_batch_upload_host(senga_batch* b, int ibox, const double* fields, const double* trun, const int32_t* itn) {
  if (!b || ibox < 0 || ibox >= (int)b->members.size() || !fields || !trun || !itn)
    return fail(SENGA_ERR_ARG, "senga_batch_upload_host: bad argument");
  return guard2([&] {
    b->ens.upload(b->members[ibox], fields, trun, itn);
    CKE(cudaStreamSynchronize(b->ens.stream));
  });
}

int senga_batch_download_host(senga_batch* b, int ibox, double* fields, double* trun, int32_t* itn) {
  if (!b || ibox < 0 || ibox >= (int)b->members.size() || !fields)
    return fail(SENGA_ERR_ARG, "senga_batch_download_host: bad argument");
  return guard2([&] {
    b->ens.download(b->members[ibox], fields, trun, itn);
    CKE(cudaStreamSynchronize(b->ens.stream));
  });
}

int senga_batch_step(senga_batch* b, int nsteps) {
  if (!b || nsteps < 0) return fail(SENGA_ERR_ARG, "senga_batch_step: bad argument");
  return guard2([&] { b->ens.step_graph(nsteps); });
}

int senga_batch_autotune(senga_batch* b, int* grid_stencil, int* grid_thermo) {
  if (!b) return fail(SENGA_ERR_ARG, "senga_batch_autotune: null batch");
  return guard2([&] {
    b->ens.autotune();
    if (grid_stencil) *grid_stencil = b->ens.grid_stencil;
    if (grid_thermo) *grid_thermo = b->ens.grid_thermo;
  });
}

int senga_batch_form(senga_batch* b, int* persistent, int* grid) {
  if (!b) return fail(SENGA_ERR_ARG, "senga_batch_form: null batch");
  if (persistent) *persistent = b->ens.persist ? 1 : 0;
  if (grid) *grid = b->ens.persist ? b->ens.grid_persist : b->ens.grid_thermo;
  return SENGA_OK;
}

int senga_batch_sync(senga_batch* b) {
  if (!b) return fail(SENGA_ERR_ARG, "senga_batch_sync: null batch");
  return guard2([&] { CKE(cudaStreamSynchronize(b->ens.stream)); });
}

void* senga_batch_stream(senga_batch* b) { return b ? (void*)b->ens.stream : nullptr; }

int senga_batch_status(senga_batch* b, int* status) {
  if (!b || !status) return fail(SENGA_ERR_ARG, "senga_batch_status: bad argument");
  return guard2([&] {
    unsigned int s = 0;
    CKE(cudaMemcpyAsync(&s, b->ens.d_status, sizeof(s), cudaMemcpyDeviceToHost, b->ens.stream));
    CKE(cudaStreamSynchronize(b->ens.stream));
    *status = (int)s;
  });
}

}  // extern "C"

// ============================================================================
// page-locked staging of the serving loop; a request's state (and result)
// may take half of it
constexpr size_t kRingBytes = size_t(4) << 30;

struct senga_server {
  Ensemble ens;
  std::map<int, Member*> all;  // every request ever submitted, by id
  std::deque<Member*> pending;  // waiting for arena room, in arrival order
  int next_id = 0;
  int64_t gpsu_done = 0;
  double t0 = 0.0;
  int64_t max_points = 0;  // admission cap on the grid points advanced per tick (0: arena only)
  PinnedRing ring;         // page-locked staging of every copy the loop makes
  int64_t finishing_points = 0;  // points of requests whose results are still on the way
  int finishing = 0, observed = 0;
  cudaEvent_t step_ev[2] = {};  // the last two steps queued: at most two run ahead
  int64_t steps_queued = 0;
};

extern "C" {

int senga_server_create(size_t arena_bytes, const senga_chem* chem, const senga_diff* diff, int device,
                        senga_server** out) {
  if (!chem || !out || arena_bytes < (1u << 20)) return fail(SENGA_ERR_ARG, "senga_server_create: bad argument");
  *out = nullptr;
  senga_server* s = new senga_server();
  int rc = guard2([&] {
    s->ens.init(*chem, diff, device, arena_bytes);
    s->ring.init(kRingBytes);
    s->t0 = now_s();
  });
  if (rc != SENGA_OK) {
    s->ens.destroy();
    s->ring.release_all();
    delete s;
    return rc;
  }
  *out = s;
  return SENGA_OK;
}

int senga_server_set_max_points(senga_server* s, int64_t max_points) {
  if (!s || max_points < 0) return fail(SENGA_ERR_ARG, "senga_server_set_max_points: bad argument");
  s->max_points = max_points;
  return SENGA_OK;
}

int senga_server_destroy(senga_server* s) {
  if (!s) return SENGA_OK;
  s->ens.destroy();
  s->ring.release_all();
  for (auto& kv : s->all) delete kv.second;
  delete s;
  return SENGA_OK;
}

int senga_server_submit(senga_server* s, const senga_config* cfg, const double* fields, const double* trun,
                        const int32_t* itn, int nsteps, int* request_id) {
  if (!s || !cfg || !fields || !trun || !itn || nsteps < 1 || !request_id)
    return fail(SENGA_ERR_ARG, "senga_server_submit: bad argument");
  return guard2([&] {
    check_box(*cfg);
    if (box_bytes(*cfg, s->ens.nspec) > s->ens.arena.capacity())
      throw Error(SENGA_ERR_NOMEM, "senga_server_submit: request larger than the arena");
    const size_t state_bytes = (size_t)cfg->nx * cfg->ny * cfg->nz * ((6 + s->ens.nspec) * sizeof(double) + 4);
    if (2 * state_bytes > kRingBytes)
      throw Error(SENGA_ERR_NOMEM, "senga_server_submit: request larger than half the page-locked staging");
    Member* m = new Member();
    m->id = s->next_id++;
    m->cfg = *cfg;
    m->steps_left = nsteps;
    m->t_submit = now_s() - s->t0;
    const int64_t n = (int64_t)cfg->nx * cfg->ny * cfg->nz;
    m->h_fields.assign(fields, fields + (size_t)(5 + s->ens.nspec) * n);
    m->h_t.assign(trun, trun + n);
    m->h_itn.assign(itn, itn + n);
    s->all[m->id] = m;
    s->pending.push_back(m);
    *request_id = m->id;
  });
}

// One serving tick: admit pending requests in arrival order while the arena
// has room, advance every active request one RK step, retire finished ones
// (copy back, free their memory). *finished receives the number retired.
int senga_server_tick(senga_server* s, int* finished) {
  if (!s) return fail(SENGA_ERR_ARG, "senga_server_tick: null server");
  return guard2([&] {
    Ensemble& E = s->ens;
    const int before = s->observed;
    s->ring.reclaim();  // results that have arrived
    bool changed = false;
    int64_t active_points = s->finishing_points;
    for (const Member* a : E.active) active_points += a->desc.g.n;
    while (!s->pending.empty()) {
      Member* m = s->pending.front();
      const int64_t n = (int64_t)m->cfg.nx * m->cfg.ny * m->cfg.nz;
      // the cap keeps a tick short, so requests run to completion in arrival
      // order instead of all sharing a slow tick; one request always fits
      if (s->max_points > 0 && active_points > 0 && active_points + n > s->max_points) break;
      if (!E.place(*m)) break;  // admission by HBM footprint, first come first served
      active_points += n;
      // the initial state through a page-locked chunk: the copy is queued
      // behind the kernels already on the stream, the host does not wait
      const size_t fb = m->h_fields.size() * sizeof(double), tb = m->h_t.size() * sizeof(double);
      const size_t ib = m->h_itn.size() * sizeof(int32_t);
      PinnedRing::Chunk* c = s->ring.take(fb + tb + ib);
      char* hp = s->ring.ptr(c);
      std::memcpy(hp, m->h_fields.data(), fb);
      std::memcpy(hp + fb, m->h_t.data(), tb);
      std::memcpy(hp + fb + tb, m->h_itn.data(), ib);
      E.upload(*m, reinterpret_cast<const double*>(hp), reinterpret_cast<const double*>(hp + fb),
               reinterpret_cast<const int32_t*>(hp + fb + tb));
      CKE(cudaEventRecord(c->ev, E.stream));
      m->t_admit = now_s() - s->t0;
      E.active.push_back(m);
      s->pending.pop_front();
      changed = true;
    }
    if (changed) E.rebuild(&s->ring);
    if (!E.active.empty()) {
      // at most two steps in flight ahead of the host
      cudaEvent_t& ev = s->step_ev[s->steps_queued & 1];
      if (!ev) CKE(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      else if (s->steps_queued >= 2) CKE(cudaEventSynchronize(ev));
      E.step_direct();
      CKE(cudaEventRecord(ev, E.stream));
      ++s->steps_queued;
      std::vector<Member*> keep;
      std::vector<Member*> fin;
      for (Member* m : E.active) {
        m->steps_left -= 1;
        m->steps_done += 1;
        s->gpsu_done += 5 * m->desc.g.n;
        (m->steps_left > 0 ? keep : fin).push_back(m);
      }
      for (Member* m : fin) {
        // the result through a page-locked chunk, copied out on the host
        // once the download has completed; the arena room is reused in
        // stream order
        const size_t fb = m->h_fields.size() * sizeof(double), tb = m->h_t.size() * sizeof(double);
        const size_t ib = m->h_itn.size() * sizeof(int32_t);
        PinnedRing::Chunk* c = s->ring.take(fb + tb + ib);
        char* hp = s->ring.ptr(c);
        E.download(*m, reinterpret_cast<double*>(hp), reinterpret_cast<double*>(hp + fb),
                   reinterpret_cast<int32_t*>(hp + fb + tb));
        CKE(cudaEventRecord(c->ev, E.stream));
        const int64_t n = m->desc.g.n;
        m->finishing = true;
        s->finishing_points += n;
        s->finishing += 1;
        c->done = [s, m, fb, tb, ib, n](const char* p) {
          std::memcpy(m->h_fields.data(), p, fb);
          std::memcpy(m->h_t.data(), p + fb, tb);
          std::memcpy(m->h_itn.data(), p + fb + tb, ib);
          m->t_done = now_s() - s->t0;
          m->finishing = false;
          s->finishing_points -= n;
          s->finishing -= 1;
          s->observed += 1;
        };
        E.unplace(*m);
      }
      if (!fin.empty()) {
        E.active = keep;
        E.rebuild(&s->ring);
      }
    } else if (s->finishing > 0) {
      s->ring.wait_oldest();  // nothing to run: wait for results on the way
    }
    s->ring.reclaim();
    if (finished) *finished = s->observed - before;
  });
}

// Result and timing of one request: state (nc interior arrays), T, ITNDEX,
// and times [submit, admit, done] in seconds since server creation. Returns
// SENGA_ERR_ARG while the request is not finished.
int senga_server_result(senga_server* s, int request_id, double* fields, double* trun, int32_t* itn, double* times) {
  if (!s) return fail(SENGA_ERR_ARG, "senga_server_result: null server");
  auto it = s->all.find(request_id);
  if (it == s->all.end()) return fail(SENGA_ERR_ARG, "senga_server_result: unknown request");
  Member* m = it->second;
  if (m->steps_left > 0 || m->finishing || m->t_done == 0.0)
    return fail(SENGA_ERR_ARG, "senga_server_result: not finished");
  if (fields) std::memcpy(fields, m->h_fields.data(), m->h_fields.size() * sizeof(double));
  if (trun) std::memcpy(trun, m->h_t.data(), m->h_t.size() * sizeof(double));
  if (itn) std::memcpy(itn, m->h_itn.data(), m->h_itn.size() * sizeof(int32_t));
  if (times) {
    times[0] = m->t_submit;
    times[1] = m->t_admit;
    times[2] = m->t_done;
  }
  return SENGA_OK;
}

// active/pending counts, grid-point substage updates so far, arena free bytes
int senga_server_stats(senga_server* s, int* active, int* pending, int64_t* gpsu, int64_t* free_bytes) {
  if (!s) return fail(SENGA_ERR_ARG, "senga_server_stats: null server");
  // requests whose results are still on the way count as active
  if (active) *active = (int)s->ens.active.size() + s->finishing;
  if (pending) *pending = (int)s->pending.size();
  if (gpsu) *gpsu = s->gpsu_done;
  if (free_bytes) *free_bytes = (int64_t)s->ens.arena.free_bytes();
  return SENGA_OK;
}

}  // extern "C"
