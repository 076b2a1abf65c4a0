// Mixed-shape batches: host planning for the persistent 5G NR int8 kernel.
//
// A plan is built once per batch layout (the list of codewords with their base
// graph, lifting size, filler count, input and output offsets).  It groups codewords
// of equal shape into work items of `tile` codewords (default: as many as one CTA
// holds; a tuner may choose smaller tiles per shape), orders items by
// decreasing work so the longest start first, and uploads the items, the per-codeword
// records and the shift / column-base tables of every (BG, Z) used.  With app_clamp
// >= 7874 the items go to the paired kernel (two codewords per 32-bit word,
// nr_pair_kernels.cu: its tensor-memory form, two CTAs per SM, when no codeword reports
// hard decisions past its core columns), otherwise to the one-codeword-per-thread
// kernel (nr_kernels.cu).  decode() zeroes
// the device work counter and launches one CTA per SM; with use_graph the two
// operations are captured once into a CUDA graph and replayed.
#include "mixed.h"

#include <algorithm>
#include <map>
#include <utility>

#include "graph.h"
#include "nr_kernels.h"

namespace syn {

namespace {

const int kLiftingSizes[kMixLiftSizes] = {2,  3,  4,  5,  6,  7,   8,   9,   10,  11,  12,  13,  14,
                                          15, 16, 18, 20, 22, 24,  26,  28,  30,  32,  36,  40,  44,
                                          48, 52, 56, 60, 64, 72,  80,  88,  96,  104, 112, 120, 128,
                                          144, 160, 176, 192, 208, 224, 240, 256, 288, 320, 352, 384};

int lifting_index(int z) {
  for (int i = 0; i < kMixLiftSizes; ++i)
    if (kLiftingSizes[i] == z) return i;
  return -1;
}

}  // namespace

MixedPlan::~MixedPlan() { release(); }

void MixedPlan::release() {
  if (exec_) cudaGraphExecDestroy(exec_);
  exec_ = nullptr;
  cudaFree(d_items_);
  cudaFree(d_cws_);
  cudaFree(d_queue_);
  cudaFree(d_shift_);
  cudaFree(d_colz_);
  d_items_ = nullptr;
  d_cws_ = nullptr;
  d_queue_ = nullptr;
  d_shift_ = nullptr;
  d_colz_ = nullptr;
}

bool MixedPlan::init(const std::vector<MixedCodeword>& cws, int beta_q, int app_clamp, int iterations,
                     const std::vector<TileHint>& hints, std::string* err) {
  auto fail = [&](const std::string& m) {
    if (err) *err = m;
    return false;
  };
  if (app_clamp < 255) return fail("app_clamp below 255 is not supported by the mixed-batch kernel");
  if (iterations < 0) return fail("iterations must be non-negative");
  std::map<std::pair<int, int>, int> tile_of;
  for (const TileHint& h : hints) tile_of[{h.bg, h.z}] = h.tile;
  // group codewords by shape
  std::map<std::pair<int, int>, std::vector<int>> groups;
  long long need_llr = 0, need_out = 0;
  for (size_t i = 0; i < cws.size(); ++i) {
    const MixedCodeword& c = cws[i];
    if (c.bg != 0 && c.bg != 1) return fail("base_graph must be 0 or 1");
    if (lifting_index(c.z) < 0) return fail("z is not a valid 3GPP lifting size");
    const long long n = (long long)(c.bg == 0 ? 68 : 52) * c.z;
    if (c.hard_bits < 0 || c.hard_bits > n) return fail("hard_bits out of range");
    if (c.n_filler < 0 || c.llr_offset < 0 || c.out_offset < 0) return fail("negative offset or filler count");
    need_llr = std::max(need_llr, c.llr_offset + n - 2LL * c.z);
    need_out = std::max(need_out, c.out_offset + (c.hard_bits + 31) / 32);
    groups[{c.bg, c.z}].push_back((int)i);
  }
  // two codewords per 32-bit word when no non-filler posterior can reach the clamp
  const bool paired = app_clamp >= 7874;
  bool core_only = true;  // every codeword's reported bits lie in its core columns
  for (const MixedCodeword& c : cws)
    if (c.hard_bits > (long long)pair_mixed_core_columns(c.bg) * c.z) core_only = false;
  std::vector<MixItem> items;
  std::vector<MixCodeword> recs;
  recs.reserve(cws.size());
  for (auto& kv : groups) {
    const int bg = kv.first.first, z = kv.first.second;
    const int cap = paired ? pair_mixed_capacity(bg, z) : mixed_slot_capacity(bg, z);
    int tile = cap;
    auto it = tile_of.find(kv.first);
    if (it != tile_of.end()) tile = std::max(1, std::min(cap, it->second));
    const std::vector<int>& idx = kv.second;
    for (size_t s = 0; s < idx.size(); s += tile) {
      MixItem m{};
      m.bg = bg;
      m.z = z;
      m.zi = lifting_index(z);
      m.count = (int)std::min<size_t>(tile, idx.size() - s);
      m.first = (int)recs.size();
      for (int j = 0; j < m.count; ++j) {
        const MixedCodeword& c = cws[idx[s + j]];
        MixCodeword r{};
        r.llr_off = c.llr_offset;
        r.out_off = c.out_offset;
        r.n_filler = c.n_filler;
        r.hard_bits = c.hard_bits;
        r.index = idx[s + j];
        recs.push_back(r);
      }
      items.push_back(m);
    }
  }
  // longest items first (edges x z x codewords), so the tail of the queue is short work
  auto cost = [](const MixItem& m) { return (long long)(m.bg == 0 ? 316 : 197) * m.z * m.count; };
  std::stable_sort(items.begin(), items.end(), [&](const MixItem& a, const MixItem& b) { return cost(a) > cost(b); });
  // shift and column-base tables of every shape in the batch
  std::vector<short> shift((size_t)2 * kMixLiftSizes * kMixEdges, 0);
  std::vector<int> colz((size_t)2 * kMixLiftSizes * kMixEdges, 0);
  for (auto& kv : groups) {
    const int bg = kv.first.first, z = kv.first.second, zi = lifting_index(z);
    Graph g;
    if (!build_nr_graph(bg, z, &g) || !nr_layout_matches(bg, g.cols.data(), g.edges()))
      return fail("internal: base graph layout mismatch");
    short* sh = &shift[((size_t)bg * kMixLiftSizes + zi) * kMixEdges];
    int* cz = &colz[((size_t)bg * kMixLiftSizes + zi) * kMixEdges];
    for (int e = 0; e < g.edges(); ++e) sh[e] = (short)g.shifts[e];
    mixed_column_bases(bg, z, cz);
  }
  release();
  need_llr_ = need_llr;
  need_out_ = need_out;
  n_items_ = (int)items.size();
  n_codewords_ = (int)cws.size();
  beta_q_ = beta_q;
  app_clamp_ = app_clamp;
  iterations_ = iterations;
  if (cudaGetDevice(&device_) != cudaSuccess) return fail("no CUDA device");
  cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, device_);
  paired_ = paired;
  tmem_ = paired && core_only;
  if ((paired ? pair_mixed_prepare() : mixed_kernel_prepare()) != cudaSuccess ||
      (tmem_ && pair_tm_mixed_prepare() != cudaSuccess))
    return fail("cannot configure the mixed-batch kernel");
  if (cudaMalloc(&d_items_, sizeof(MixItem) * std::max<size_t>(items.size(), 1)) != cudaSuccess ||
      cudaMalloc(&d_cws_, sizeof(MixCodeword) * std::max<size_t>(recs.size(), 1)) != cudaSuccess ||
      cudaMalloc(&d_queue_, sizeof(unsigned)) != cudaSuccess ||
      cudaMalloc(&d_shift_, sizeof(short) * shift.size()) != cudaSuccess ||
      cudaMalloc(&d_colz_, sizeof(int) * colz.size()) != cudaSuccess) {
    release();
    return fail("cudaMalloc failed for the plan tables");
  }
  cudaMemcpy(d_items_, items.data(), sizeof(MixItem) * items.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(d_cws_, recs.data(), sizeof(MixCodeword) * recs.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(d_shift_, shift.data(), sizeof(short) * shift.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(d_colz_, colz.data(), sizeof(int) * colz.size(), cudaMemcpyHostToDevice);
  items_ = items;
  if (cudaGetLastError() != cudaSuccess) return fail("copying the plan tables failed");
  return true;
}

bool MixedPlan::set_kernel(int kernel) {
  if (kernel != 0 && kernel != 5) return false;
  if (kernel != kernel_ && exec_) {  // a captured graph holds the other kernel
    cudaGraphExecDestroy(exec_);
    exec_ = nullptr;
  }
  kernel_ = kernel;
  return true;
}

MixArgs MixedPlan::args(const int8_t* d_llr, uint32_t* d_out, int32_t* d_iters) const {
  MixArgs m{};
  m.items = d_items_;
  m.n_items = n_items_;
  m.cws = d_cws_;
  m.llr = d_llr;
  m.out = d_out;
  m.iters = d_iters;
  m.shift_tab = d_shift_;
  m.colz_tab = d_colz_;
  m.queue = d_queue_;
  m.beta_q = beta_q_;
  m.app_clamp = app_clamp_;
  m.iterations = iterations_;
  m.k32 = 32;
  m.two = 2;
  return m;
}

cudaError_t MixedPlan::decode(const int8_t* d_llr, uint32_t* d_out, int32_t* d_iters, bool use_graph,
                              cudaStream_t stream) {
  if (n_items_ == 0) return cudaSuccess;
  const MixArgs m = args(d_llr, d_out, d_iters);
  auto launch = [&](cudaStream_t st) {
    if (tmem_ && kernel_ != 5) return pair_tm_mixed_launch(m, sms_, st);
    return paired_ ? pair_mixed_launch(m, sms_, st) : mixed_decode_launch(m, sms_, st);
  };
  if (!use_graph) return launch(stream);
  if (!exec_ || g_llr_ != d_llr || g_out_ != d_out || g_iters_ != d_iters) {
    if (exec_) cudaGraphExecDestroy(exec_);
    exec_ = nullptr;
    cudaStream_t cap = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
    if (e != cudaSuccess) return e;
    cudaGraph_t graph = nullptr;
    e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      const cudaError_t le = launch(cap);
      e = cudaStreamEndCapture(cap, &graph);
      if (le != cudaSuccess) e = le;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec_, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    cudaStreamDestroy(cap);
    if (e != cudaSuccess) {
      exec_ = nullptr;
      return e;
    }
    g_llr_ = d_llr;
    g_out_ = d_out;
    g_iters_ = d_iters;
  }
  return cudaGraphLaunch(exec_, stream);
}

}  // namespace syn
