#include <cmath>
// Batched rendering: several scenes (built contexts) rendered by one wavefront pass.  No counterpart
// in the reference, which renders one scene per OptiX launch (OptixScene::renderScene,
// OptixScene.cpp:139-168); every scene of a batch still follows that launch's semantics (its probe
// pass, its camera paths seeded by (pixel, frame), its running mean in frame order), so a batched
// render produces the same images as rendering the scenes one by one.
//
// The pass lays the scenes' frames out as items in one path-id space (pt_render.cu), so small scenes
// fill the GPU together instead of one after another, and the whole launch sequence of a render
// (probe passes, bounces, gathers, accumulation of every scene) is captured once into a CUDA graph
// and replayed: one graph launch per batch render.  The launch options are chosen by an autotuner
// that times short renders of the batch itself.
#include <algorithm>
#include <cstring>
#include <string>

#include "pt_context.h"

using namespace pt;

struct pt_batch {
  pt_ctx* eng = nullptr;  // engine: stream, wavefront, scene/item tables, options, statistics
  std::vector<pt_ctx*> scenes;
  std::vector<uint32_t> frames;  // frames per batch render, per scene
  bool use_graph = true;
  cudaGraphExec_t exec = nullptr;
  std::vector<uint64_t> key;     // what the captured graph depends on
  uint64_t graph_kernels = 0;    // kernel nodes of the captured graph
  cudaEvent_t done = nullptr;
};

namespace {

void drop_graph(pt_batch* b)
{
  if (b->exec) cudaGraphExecDestroy(b->exec);
  b->exec = nullptr;
  b->key.clear();
  b->graph_kernels = 0;
}

// Everything the captured launch sequence depends on: the pass layout (chunks, counts, bounces), the
// device buffers and options it was launched with, and the scene records themselves (a chunk that
// holds one scene passes its record to the traversal kernels by value, so the graph holds a copy).
// Item first frames are read from device memory at run time and may change between launches.
std::vector<uint64_t> graph_key(const Context& E, const PassLayout& L, const std::vector<SceneDev>& tab)
{
  std::vector<uint64_t> k;
  for (const SceneDev& sd : tab) {  // each record's bytes, word by word (compared exactly)
    uint64_t words[(sizeof(SceneDev) + 7) / 8] = {};
    memcpy(words, &sd, sizeof(SceneDev));
    k.insert(k.end(), words, words + (sizeof(SceneDev) + 7) / 8);
  }
  k.push_back((uint64_t)L.passes);
  k.push_back(L.sss ? 1 : 0);
  k.push_back(L.layered ? 1 : 0);
  k.push_back(L.ms ? 1 : 0);
  k.push_back(L.g_slots);
  k.push_back(L.items.size());
  for (size_t i = 0; i < L.chunk_paths.size(); ++i) {
    k.push_back(L.chunk_item_begin[i]);
    k.push_back(L.chunk_paths[i]);
    k.push_back(L.chunk_probes[i]);
    k.push_back(L.chunk_pixels[i]);
    k.push_back(L.chunk_sets[i]);
  }
  for (const void* p : {E.wf.rays.p, E.wf.state.p, E.wf.g_a.p, E.wf.probes.p, E.d_scene_tab.p, E.d_item_tab.p, E.wf.counters.p, E.wf.path_item.p,
                        E.wf2.rays.p, E.wf2.state.p, E.wf2.counters.p, E.wf2.path_item.p})
    k.push_back((uint64_t)(uintptr_t)p);
  k.push_back(E.wf.cap);
  k.push_back((uint64_t)E.opt.extend_mode);
  k.push_back((uint64_t)E.opt.refill);
  k.push_back((uint64_t)E.opt.bin_items);
  k.push_back((uint64_t)E.opt.overlap);
  k.push_back((uint64_t)E.opt.dual);
  k.push_back((uint64_t)L.dual);
  k.push_back((uint64_t)E.pass_w4);
  return k;
}

// Validates and prepares every scene, orders the engine's stream after their uploads, and plans the
// pass of frames [next_frame, next_frame + frames) of each scene.
pt_status plan(pt_batch* b, PassLayout& L, std::vector<SceneDev>& tab, uint64_t& samples, const std::vector<uint32_t>* frames_override)
{
  Context& E = b->eng->c;
  if (b->scenes.empty()) return fail(PT_NOT_READY, "pt_batch_render: the batch has no scenes");
  std::vector<SceneFacts> facts;
  std::vector<ItemReq> reqs;
  tab.clear();
  samples = 0;
  for (size_t k = 0; k < b->scenes.size(); ++k) {
    Context& c = b->scenes[k]->c;
    pt_status st = prepare_scene(c, "pt_batch_render");
    if (st != PT_OK) return st;
    PT_CHECK_CUDA(cudaEventRecord(c.ext0, c.stream), "batch order");
    PT_CHECK_CUDA(cudaStreamWaitEvent(E.stream, c.ext0, 0), "batch order");
    SceneFacts f = scene_facts(c);
    facts.push_back(f);
    uint32_t nf = frames_override ? (*frames_override)[k] : b->frames[k];
    reqs.push_back(ItemReq{(uint32_t)k, c.next_frame, nf});
    tab.push_back(c.view());
    samples += scene_path_samples(c, nf);
  }
  PT_CHECK_CUDA(cudaSetDevice(E.device), "cudaSetDevice");
  L = plan_pass(facts, reqs, E.max_paths, E.opt.dual != 0);
  return PT_OK;
}

// Orders every scene's stream after the engine's work (read-backs on a scene see the batch's result).
pt_status release(pt_batch* b)
{
  Context& E = b->eng->c;
  PT_CHECK_CUDA(cudaEventRecord(b->done, E.stream), "batch order");
  for (pt_ctx* s : b->scenes) PT_CHECK_CUDA(cudaStreamWaitEvent(s->c.stream, b->done, 0), "batch order");
  return PT_OK;
}

// One render of the batch; graph: capture / replay the launch sequence.
pt_status render(pt_batch* b, bool graph, const std::vector<uint32_t>* frames_override, bool advance)
{
  Context& E = b->eng->c;
  PassLayout L;
  std::vector<SceneDev> tab;
  uint64_t samples = 0;
  pt_status st = plan(b, L, tab, samples, frames_override);
  if (st != PT_OK) return st;
  if ((st = pass_resources(E, L, tab)) != PT_OK) return st;
  const bool multi = tab.size() > 1;
  uint64_t launches0 = pt_kernel_launch_count();
  memset(&E.stats, 0, sizeof(E.stats));
  if (graph) {
    std::vector<uint64_t> key = graph_key(E, L, tab);
    if (!b->exec || key != b->key) {
      drop_graph(b);
      cudaGraph_t g = nullptr;
      const uint64_t k0 = pt_kernel_launch_count();
      PT_CHECK_CUDA(cudaStreamBeginCapture(E.stream, cudaStreamCaptureModeThreadLocal), "graph capture");
      st = launch_pass(E, L, tab, multi, false);
      const uint64_t captured = pt_kernel_launch_count() - k0;
      cudaError_t e = cudaStreamEndCapture(E.stream, &g);
      if (st != PT_OK) {
        if (g) cudaGraphDestroy(g);
        return st;
      }
      if (e != cudaSuccess) return cuda_status(e, "graph capture");
      e = cudaGraphInstantiate(&b->exec, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) {
        b->exec = nullptr;
        return cuda_status(e, "graph instantiate");
      }
      b->key = key;
      b->graph_kernels = captured;
      launches0 += captured;  // captured, not launched
    }
    PT_CHECK_CUDA(cudaEventRecord(E.ev0, E.stream), "event");
    PT_CHECK_CUDA(cudaGraphLaunch(b->exec, E.stream), "graph launch");
    PT_CHECK_CUDA(cudaEventRecord(E.ev1, E.stream), "event");
    count_launch(b->graph_kernels);  // the graph's kernel nodes run once per launch
  } else {
    PT_CHECK_CUDA(cudaEventRecord(E.ev0, E.stream), "event");
    if ((st = launch_pass(E, L, tab, multi, true)) != PT_OK) return st;
    PT_CHECK_CUDA(cudaEventRecord(E.ev1, E.stream), "event");
  }
  E.stats.path_samples = samples;
  E.stats.kernel_launches = (uint32_t)(pt_kernel_launch_count() - launches0);
  E.stats_pending = true;
  if (advance)
    for (size_t k = 0; k < b->scenes.size(); ++k)
      b->scenes[k]->c.next_frame += frames_override ? (*frames_override)[k] : b->frames[k];
  return release(b);
}

}  // namespace

extern "C" {

pt_status pt_batch_create(int device, pt_batch** out)
{
  if (!out) return fail(PT_INVALID_ARG, "pt_batch_create: null output");
  *out = nullptr;
  pt_batch* b = new (std::nothrow) pt_batch();
  if (!b) return fail(PT_OOM, "pt_batch_create: host allocation");
  pt_status st = pt_context_create(device, &b->eng);
  if (st != PT_OK) {
    delete b;
    return st;
  }
  cudaError_t e = cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    pt_context_destroy(b->eng);
    delete b;
    return cuda_status(e, "pt_batch_create");
  }
  *out = b;
  return PT_OK;
}

pt_status pt_batch_destroy(pt_batch* b)
{
  if (!b) return PT_OK;
  cudaSetDevice(b->eng->c.device);
  cudaStreamSynchronize(b->eng->c.stream);
  drop_graph(b);
  if (b->done) cudaEventDestroy(b->done);
  pt_context_destroy(b->eng);
  delete b;
  return PT_OK;
}

void* pt_batch_stream(pt_batch* b) { return b ? (void*)b->eng->c.stream : nullptr; }

pt_status pt_batch_add(pt_batch* b, pt_ctx* scene, uint32_t frames_per_render)
{
  if (!b || !scene) return fail(PT_INVALID_ARG, "pt_batch_add: null argument");
  if (scene->c.device != b->eng->c.device) return fail(PT_INVALID_ARG, "pt_batch_add: the scene lives on another device");
  if (frames_per_render == 0) return fail(PT_INVALID_ARG, "pt_batch_add: frames_per_render must be >= 1");
  if (b->scenes.size() >= 65535) return fail(PT_CAP_EXCEEDED, "pt_batch_add: at most 65535 scenes");
  for (pt_ctx* s : b->scenes)
    if (s == scene) return fail(PT_INVALID_ARG, "pt_batch_add: scene already in the batch");
  b->scenes.push_back(scene);
  b->frames.push_back(frames_per_render);
  drop_graph(b);
  return PT_OK;
}

pt_status pt_batch_set_option(pt_batch* b, const char* name, int64_t value)
{
  if (!b || !name) return fail(PT_INVALID_ARG, "pt_batch_set_option: null argument");
  std::string k(name);
  drop_graph(b);
  if (k == "use_graph") {
    if (value != 0 && value != 1) return fail(PT_INVALID_ARG, "pt_batch_set_option: use_graph must be 0 or 1");
    b->use_graph = value != 0;
    return PT_OK;
  }
  if (k == "max_paths_in_flight") return pt_set_max_paths_in_flight(b->eng, (uint64_t)value);
  if (k == "profile") return pt_set_profiling(b->eng, (int)value);
  return pt_set_option(b->eng, name, value);
}

pt_status pt_batch_render(pt_batch* b)
{
  if (!b) return fail(PT_INVALID_ARG, "pt_batch_render: null batch");
  return render(b, b->use_graph, nullptr, true);
}

pt_status pt_batch_render_sequential(pt_batch* b)
{
  if (!b) return fail(PT_INVALID_ARG, "pt_batch_render_sequential: null batch");
  if (b->scenes.empty()) return fail(PT_NOT_READY, "pt_batch_render_sequential: the batch has no scenes");
  Context& E = b->eng->c;
  // the plain path: every scene rendered by itself, one pass after the other, on the engine's buffers
  uint64_t launches0 = pt_kernel_launch_count(), samples = 0;
  std::vector<PassLayout> layouts;
  std::vector<SceneDev> one(1);
  pt_render_stats total;
  memset(&total, 0, sizeof(total));
  for (size_t k = 0; k < b->scenes.size(); ++k) {
    Context& c = b->scenes[k]->c;
    pt_status st = prepare_scene(c, "pt_batch_render_sequential");
    if (st != PT_OK) return st;
    PT_CHECK_CUDA(cudaEventRecord(c.ext0, c.stream), "batch order");
    PT_CHECK_CUDA(cudaStreamWaitEvent(E.stream, c.ext0, 0), "batch order");
  }
  PT_CHECK_CUDA(cudaSetDevice(E.device), "cudaSetDevice");
  PT_CHECK_CUDA(cudaEventRecord(E.ev0, E.stream), "event");
  for (size_t k = 0; k < b->scenes.size(); ++k) {
    Context& c = b->scenes[k]->c;
    SceneFacts f = scene_facts(c);
    PassLayout L = plan_pass({f}, {ItemReq{0, c.next_frame, b->frames[k]}}, E.max_paths, E.opt.dual != 0);
    one[0] = c.view();
    pt_status st = pass_resources(E, L, one);
    if (st == PT_OK) st = launch_pass(E, L, one, false, false);
    if (st != PT_OK) return st;
    samples += scene_path_samples(c, b->frames[k]);
    c.next_frame += b->frames[k];
  }
  PT_CHECK_CUDA(cudaEventRecord(E.ev1, E.stream), "event");
  E.stats = total;
  E.stats.path_samples = samples;
  E.stats.kernel_launches = (uint32_t)(pt_kernel_launch_count() - launches0);
  E.stats_pending = true;
  return release(b);
}

pt_status pt_batch_get_stats(pt_batch* b, pt_render_stats* out)
{
  if (!b) return fail(PT_INVALID_ARG, "pt_batch_get_stats: null batch");
  return pt_get_render_stats(b->eng, out);
}

pt_status pt_batch_autotune(pt_batch* b, uint32_t frames_per_trial, pt_tune_result* out)
{
  if (!b || !out) return fail(PT_INVALID_ARG, "pt_batch_autotune: null argument");
  if (frames_per_trial == 0) return fail(PT_INVALID_ARG, "pt_batch_autotune: frames_per_trial must be >= 1");
  if (b->scenes.empty()) return fail(PT_NOT_READY, "pt_batch_autotune: the batch has no scenes");
  Context& E = b->eng->c;
  std::vector<uint32_t> saved_next;
  for (pt_ctx* s : b->scenes) saved_next.push_back(s->c.next_frame);
  std::vector<uint32_t> trial_frames;
  for (uint32_t f : b->frames) trial_frames.push_back(std::min(f, frames_per_trial));
  const Options saved_opt = E.opt;
  const uint64_t saved_max = E.max_paths;
  struct Cand { int mode, refill; uint64_t max_paths; };
  std::vector<Cand> cands;
  for (uint64_t mp : {1ull << 22, 1ull << 23, 1ull << 24})
    for (int r : {16, 20, 24}) cands.push_back({1, r, mp});
  cands.push_back({0, 20, 1ull << 23});
  float best = 0.0f;
  Cand win = cands.front();
  uint32_t trials = 0;
  for (const Cand& cd : cands) {
    E.opt.extend_mode = cd.mode;
    E.opt.refill = cd.refill;
    E.max_paths = cd.max_paths;
    for (size_t k = 0; k < b->scenes.size(); ++k) b->scenes[k]->c.next_frame = 0;
    pt_status st = render(b, false, &trial_frames, false);  // warm (allocations, caches)
    if (st == PT_OK) st = render(b, false, &trial_frames, false);
    if (st != PT_OK) return st;
    PT_CHECK_CUDA(cudaStreamSynchronize(E.stream), "autotune");
    float ms = 0.0f;
    PT_CHECK_CUDA(cudaEventElapsedTime(&ms, E.ev0, E.ev1), "autotune timing");
    float rate = ms > 0.0f ? (float)E.stats.path_samples / ms : 0.0f;
    ++trials;
    if (rate > best) {
      best = rate;
      win = cd;
    }
  }
  // second stage: the sort granularity (queue positions per binning thread) for the winner
  int win_items = E.opt.bin_items;
  E.opt.extend_mode = win.mode;
  E.opt.refill = win.refill;
  E.max_paths = win.max_paths;
  for (int items : {4, 16}) {
    if (items == win_items) continue;
    E.opt.bin_items = items;
    for (size_t k = 0; k < b->scenes.size(); ++k) b->scenes[k]->c.next_frame = 0;
    pt_status st = render(b, false, &trial_frames, false);
    if (st == PT_OK) st = render(b, false, &trial_frames, false);
    if (st != PT_OK) return st;
    PT_CHECK_CUDA(cudaStreamSynchronize(E.stream), "autotune");
    float ms = 0.0f;
    PT_CHECK_CUDA(cudaEventElapsedTime(&ms, E.ev0, E.ev1), "autotune timing");
    const float rate = ms > 0.0f ? (float)E.stats.path_samples / ms : 0.0f;
    ++trials;
    if (rate > best) {
      best = rate;
      win_items = items;
    }
  }
  E.opt = saved_opt;
  E.opt.extend_mode = win.mode;
  E.opt.refill = win.refill;
  E.opt.bin_items = win_items;
  E.max_paths = win.max_paths;
  (void)saved_max;
  drop_graph(b);
  // the trials rendered from frame 0: every scene's accumulation restarts at frame 0
  for (pt_ctx* s : b->scenes) s->c.next_frame = 0;
  (void)saved_next;
  out->extend_mode = win.mode;
  out->refill = win.refill;
  out->max_paths_in_flight = win.max_paths;
  out->best_mpaths_per_s = best / 1e3f;
  out->trials = trials;
  out->bin_items = (uint32_t)win_items;
  return PT_OK;
}

pt_status pt_get_next_frame(pt_ctx* ctx, uint32_t* out)
{
  if (!ctx || !out) return fail(PT_INVALID_ARG, "pt_get_next_frame: null argument");
  *out = ctx->c.next_frame;
  return PT_OK;
}

pt_status pt_set_accumulation(pt_ctx* ctx, const float* host_rgba, uint32_t next_frame)
{
  if (!ctx || !host_rgba) return fail(PT_INVALID_ARG, "pt_set_accumulation: null argument");
  Context& c = ctx->c;
  if (!c.camera_set) return fail(PT_NOT_READY, "pt_set_accumulation: camera not set");
  const size_t n = (size_t)c.cam.width * c.cam.height * 4;
  for (size_t k = 0; k < n; ++k)
    if (!std::isfinite(host_rgba[k])) return fail(PT_INVALID_ARG, "pt_set_accumulation: non-finite value");
  PT_CHECK_CUDA(cudaSetDevice(c.device), "cudaSetDevice");
  PT_CHECK_CUDA(cudaMemcpyAsync(c.d_accum.p, host_rgba, n * sizeof(float), cudaMemcpyHostToDevice, c.stream), "pt_set_accumulation");
  PT_CHECK_CUDA(cudaStreamSynchronize(c.stream), "pt_set_accumulation");
  c.next_frame = next_frame;
  return PT_OK;
}

}  // extern "C"
