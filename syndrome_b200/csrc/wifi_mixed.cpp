// Host plan of a mixed batch of 802.11 codewords for the persistent f32 kernel
// (wifi_mixed.h; kernel in ldpc_kernels.cu).
//
// A plan is built once per batch layout: the codewords are grouped by matrix, the
// matrices ordered by decreasing work per codeword (edges x Z) so that the long
// codewords start first, and each matrix's codewords cut into chunks (by default about
// four per CTA over the batch, at least four codewords).  The matrices' edge and layer tables, the per-codeword records and
// the chunk list go to the device once; decode() zeroes the device chunk counter and
// launches the persistent kernel with as many CTAs as the SMs hold, optionally from a
// captured CUDA graph.
#include "wifi_mixed.h"

#include <algorithm>
#include <map>
#include <tuple>

#include "graph.h"

namespace syn {

namespace {

int maxdeg_class(int maxdeg) {
  if (maxdeg <= 8) return 8;
  if (maxdeg <= 12) return 12;
  if (maxdeg <= 16) return 16;
  if (maxdeg <= 24) return 24;
  return -1;
}

}  // namespace

WifiMixedPlan::~WifiMixedPlan() { release(); }

void WifiMixedPlan::release() {
  if (exec_) cudaGraphExecDestroy(exec_);
  exec_ = nullptr;
  cudaFree(d_shapes_);
  cudaFree(d_edges_);
  cudaFree(d_loffs_);
  cudaFree(d_cws_);
  cudaFree(d_chunks_);
  cudaFree(d_queue_);
  d_shapes_ = nullptr;
  d_edges_ = nullptr;
  d_loffs_ = nullptr;
  d_cws_ = nullptr;
  d_chunks_ = nullptr;
  d_queue_ = nullptr;
}

bool WifiMixedPlan::init(const std::vector<WifiMixedCodeword>& cws, float beta, int iterations, int chunk,
                         std::string* err) {
  auto fail = [&](const std::string& m) {
    if (err) *err = m;
    return false;
  };
  if (iterations < 0) return fail("iterations must be non-negative");
  if (chunk < 0) return fail("chunk must be non-negative");
  using Key = std::tuple<int, int, int>;
  std::map<Key, std::vector<int>> groups;
  std::map<Key, Graph> graphs;
  long long need_llr = 0, need_out = 0;
  for (size_t i = 0; i < cws.size(); ++i) {
    const WifiMixedCodeword& c = cws[i];
    const Key key{c.z, c.rate_num, c.rate_den};
    if (!graphs.count(key)) {
      Graph g;
      if (!build_wifi_graph(c.z, c.rate_num, c.rate_den, &g))
        return fail("not an 802.11 matrix: z must be 27, 54 or 81 and the rate 1/2, 2/3, 3/4 or 5/6");
      if (maxdeg_class(g.maxdeg) < 0 || g.edges() > kWmMaxEdges || g.mb > kWmMaxLayers)
        return fail("internal: matrix larger than the kernel's tables");
      graphs[key] = g;
    }
    const long long n = graphs[key].n();
    if (c.hard_bits < 0 || c.hard_bits > n) return fail("hard_bits out of range");
    if (c.llr_offset < 0 || c.out_offset < 0) return fail("negative offset");
    need_llr = std::max(need_llr, c.llr_offset + n);
    need_out = std::max(need_out, c.out_offset + (c.hard_bits + 31) / 32);
    groups[key].push_back((int)i);
  }
  // matrices by decreasing work per codeword
  std::vector<Key> order;
  for (auto& kv : groups) order.push_back(kv.first);
  std::stable_sort(order.begin(), order.end(), [&](const Key& x, const Key& y) {
    return (long long)graphs[x].edges() * graphs[x].z > (long long)graphs[y].edges() * graphs[y].z;
  });
  // Default chunk: about four per CTA over the whole batch (two CTAs per SM), at least
  // four codewords (or a CTA's slots, if fewer): enough chunks that the CTAs finish
  // together, few enough that a CTA rarely switches matrices (a sweep over 32,768
  // codewords: 16-32 codewords per chunk 3.95-4.00 Gbit/s, 8 3.77, 64 3.47, the earlier
  // default of four CTAs' slots 3.65; 1,024 codewords of one matrix, Z = 27: 4 per
  // chunk 0.197 ms, 14 0.234 ms).
  int dev = 0, sms_now = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms_now, cudaDevAttrMultiProcessorCount, dev);
  const long long even = ((long long)cws.size() + 8LL * sms_now - 1) / (8LL * std::max(sms_now, 1));
  std::vector<WmShape> shapes;
  std::vector<uint32_t> edges;
  std::vector<int32_t> loffs;
  std::vector<WmCodeword> recs;
  std::vector<WmChunk> chunks;
  int smem = 0;
  for (const Key& key : order) {
    const Graph& g = graphs[key];
    WmShape s{};
    s.z = g.z;
    s.n = (int)g.n();
    s.mb = g.mb;
    s.n_edges = g.edges();
    s.cpb = std::min(kWmMaxSlots, kWmThreads / g.z);
    s.st_words = 2 * g.mb;
    for (int l = 0; l < g.mb; ++l) s.st_words += std::max(1, (g.layer_off[l + 1] - g.layer_off[l] + 15) / 16);
    s.maxdeg_tmpl = maxdeg_class(g.maxdeg);
    s.edge_off = (int)edges.size();
    s.loff_off = (int)loffs.size();
    for (int e = 0; e < g.edges(); ++e) edges.push_back(((uint32_t)(g.cols[e] * g.z) << 16) | (uint32_t)g.shifts[e]);
    for (int l = 0; l <= g.mb; ++l) loffs.push_back(g.layer_off[l]);
    smem = std::max(smem, wifi_mixed_smem_bytes(s));
    const int shape = (int)shapes.size();
    shapes.push_back(s);
    const int per_chunk = chunk > 0 ? chunk : (int)std::max<long long>(std::min(s.cpb, 4), even);
    const std::vector<int>& idx = groups[key];
    for (size_t f = 0; f < idx.size(); f += per_chunk) {
      WmChunk ch{};
      ch.shape = shape;
      ch.first = (int)recs.size();
      ch.count = (int)std::min<size_t>(per_chunk, idx.size() - f);
      for (int j = 0; j < ch.count; ++j) {
        const WifiMixedCodeword& c = cws[idx[f + j]];
        WmCodeword r{};
        r.llr_off = c.llr_offset;
        r.out_off = c.out_offset;
        r.hard_bits = c.hard_bits;
        r.index = idx[f + j];
        recs.push_back(r);
      }
      chunks.push_back(ch);
    }
  }
  release();
  need_llr_ = need_llr;
  need_out_ = need_out;
  n_codewords_ = (int)cws.size();
  n_chunks_ = (int)chunks.size();
  iterations_ = iterations;
  beta_ = beta;
  smem_ = smem;
  if (cudaGetDevice(&device_) != cudaSuccess) return fail("no CUDA device");
  int sms = 0, per_sm = 1;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_);
  if (smem > 0 && wifi_mixed_prepare(smem, &per_sm) != cudaSuccess) return fail("cannot configure the kernel");
  ctas_ = std::max(1, sms * per_sm);
  auto up = [&](auto** dst, const auto& v) {
    using T = typename std::remove_reference<decltype(v)>::type::value_type;
    const size_t bytes = sizeof(T) * std::max<size_t>(v.size(), 1);
    if (cudaMalloc(reinterpret_cast<void**>(dst), bytes) != cudaSuccess) return false;
    return v.empty() || cudaMemcpy(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice) == cudaSuccess;
  };
  if (!up(&d_shapes_, shapes) || !up(&d_edges_, edges) || !up(&d_loffs_, loffs) || !up(&d_cws_, recs) ||
      !up(&d_chunks_, chunks) || cudaMalloc(reinterpret_cast<void**>(&d_queue_), sizeof(unsigned)) != cudaSuccess) {
    release();
    return fail("cudaMalloc / copy failed for the plan tables");
  }
  return true;
}

WmArgs WifiMixedPlan::args(const float* d_llr, uint32_t* d_out, int32_t* d_iters) const {
  WmArgs a{};
  a.shapes = d_shapes_;
  a.edges = d_edges_;
  a.loffs = d_loffs_;
  a.cws = d_cws_;
  a.chunks = d_chunks_;
  a.n_chunks = n_chunks_;
  a.llr = d_llr;
  a.out = d_out;
  a.iters = d_iters;
  a.queue = d_queue_;
  a.iterations = iterations_;
  a.beta = beta_;
  return a;
}

cudaError_t WifiMixedPlan::decode(const float* d_llr, uint32_t* d_out, int32_t* d_iters, bool use_graph,
                                  cudaStream_t stream) {
  if (n_chunks_ == 0) return cudaSuccess;
  const WmArgs a = args(d_llr, d_out, d_iters);
  if (!use_graph) return wifi_mixed_launch(a, ctas_, smem_, stream);
  if (!exec_ || g_llr_ != d_llr || g_out_ != d_out || g_iters_ != d_iters) {
    if (exec_) cudaGraphExecDestroy(exec_);
    exec_ = nullptr;
    cudaStream_t cap = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
    if (e != cudaSuccess) return e;
    cudaGraph_t graph = nullptr;
    e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      const cudaError_t le = wifi_mixed_launch(a, ctas_, smem_, cap);
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
