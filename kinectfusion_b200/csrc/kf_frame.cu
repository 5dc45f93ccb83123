// kf_frame.cu - the whole per-frame pipeline as one CUDA graph
// (Reconstruction::process_frame, reconstruction.cpp:184-277):
//   depth upload -> bilateral + 3-level pyramid -> integration pixel table ->
//   for level 2, 1, 0: [model raycast at the current estimate, one
//   cooperative kernel running the level's N Gauss-Newton steps] ->
//   integrate at the tracked pose (skipped on a tracking failure) -> result
//   download.
// One graph launch and at most one host synchronisation per frame.  The
// reference syncs once per ICP iteration (icp_correspondence.cu:589-596).
#include <cstring>
#include <map>

#include <vector>

#include "kf_internal.h"

namespace kf {
namespace {

__global__ void frame_begin_kernel(IcpState* st) {
  if (threadIdx.x != 0) return;
  // The reference keeps the camera pose as a float matrix between frames
  // (reconstruction.cpp:237-275): each frame starts from the float pose.
  for (int i = 0; i < 12; ++i) st->pose[i] = static_cast<double>(static_cast<float>(st->pose[i]));
  st->failed = 0;
  for (int l = 0; l < 4; ++l) {
    st->level_status[l] = KF_ICP_NOT_RUN;
    st->level_iterations[l] = 0;
    st->level_correspondences[l] = 0;
  }
}

}  // namespace

namespace {

// Records the frame's work on `s` (stream capture).  The frame's inputs -
// the pyramid, the integration pixel table and the depth tiles of the block
// culling - need only the depth frame, not the pose.  With `key.fork` they
// form a side branch of the graph (captured on the pipeline's side stream)
// that runs beside the coarsest level's model render and ICP, and joins
// before the first ICP step (the pyramid) and before the integration (the
// rest); without, they run first on `s`.
void record_frame(Pipeline& p, Pyramid& pyr, Tracker& t, const Pipeline::GraphKey& key, bool has_color,
                  cudaStream_t s) {
  IcpState* st = t.state.ptr;
  const bool fork = key.fork != 0;
  const cudaStream_t side = fork ? p.side_stream : s;
  if (fork) {
    check(cudaEventRecord(p.fork_event, s), "graph fork");
    check(cudaStreamWaitEvent(side, p.fork_event, 0), "graph fork");
  }
  pyr.launch(side);
  if (fork) check(cudaEventRecord(p.pyramid_event, side), "graph fork");
  const PyramidLevelBuffers& l0 = pyr.levels[0];
  const Intr k0 = intr_from(pyr.intrinsics);
  launch_pixel_table(pyr.raw.ptr, has_color ? p.frame_color.ptr : nullptr, l0.normals.ptr, pyr.width, pyr.height, k0,
                     p.config.integration, p.config.tsdf_rule, p.pixel_table.ptr, side);
  launch_integrate_inputs(p, p.pixel_table.ptr, pyr.width, pyr.height, side);
  if (fork) check(cudaEventRecord(p.inputs_event, side), "graph join");
  frame_begin_kernel<<<1, 32, 0, s>>>(st);
  check(cudaGetLastError(), "frame_begin launch");
  bool pyramid_joined = false;
  if (!key.first) {
    const uint32_t iters[4] = {key.it0, key.it1, key.it2, key.it3};
    for (int level = static_cast<int>(pyr.level_count) - 1; level >= 0; --level) {
      const PyramidLevelBuffers& b = pyr.levels[level];
      // AppOptions::raycast_camera (app_options.cpp:94-103)
      kf_raycast_camera cam;
      cam.intrinsics = b.intrinsics;
      cam.width = pyr.width >> level;
      cam.height = pyr.height >> level;
      std::memset(&cam.camera_to_world, 0, sizeof(cam.camera_to_world));
      Pipeline::Maps& m = p.maps_for(cam.width, cam.height);
      launch_raycast(p, cam, m.points.ptr, m.normals.ptr, m.colors.ptr, st, s);
      IcpLevelArgs a;
      a.live_vertices = b.vertices.ptr;
      a.live_normals = b.normals.ptr;
      a.live_width = b.width;
      a.live_height = b.height;
      a.model_points = m.points.ptr;
      a.model_normals = m.normals.ptr;
      a.model_width = cam.width;
      a.model_height = cam.height;
      a.model_intrinsics = intr_from(cam.intrinsics);
      if (fork && !pyramid_joined) {
        check(cudaStreamWaitEvent(s, p.pyramid_event, 0), "graph join");
        pyramid_joined = true;
      }
      // the level's start, steps and end in one cooperative launch; the
      // render above used the camera the previous level (or the frame
      // start) left, which is the level start's camera.  A frame graph that
      // runs beside others (a batch member) takes the same level as
      // launches that need no co-residency: cooperative launches of several
      // members could not share the GPU.
      if (key.cooperative) {
        launch_icp_level(a, st, t.partials.ptr, t.params, iters[level], level, 1, 0, s);
      } else {
        launch_icp_level_steps(a, st, t.partials.ptr, t.params, iters[level], level, s);
      }
    }
  }
  if (fork) check(cudaStreamWaitEvent(s, p.inputs_event, 0), "graph join");  // also joins the pyramid
  launch_integrate(p, p.pixel_table.ptr, pyr.width, pyr.height, k0, Rigid{}, has_color, st, s, true);
  check(cudaMemcpyAsync(p.result_staging.ptr, st, sizeof(IcpState), cudaMemcpyDeviceToHost, s), "result download");
}

// The frame graph of (pipeline, pyramid, tracker) for this frame's size,
// schedule, first-frame flag and colour, captured on first use.
Pipeline::FrameGraph& frame_graph_for(kf_pipeline* pipeline, kf_pyramid* pyramid, kf_tracker* tracker,
                                      uint32_t width, uint32_t height, kf_intrinsics intrinsics,
                                      const uint32_t* iterations, int32_t first_frame, bool has_color,
                                      bool fork = true, bool cooperative = true) {
  require(pipeline && pyramid && tracker, "kf_frame_enqueue: null argument");
  require(intrinsics.fx > 0.0f && intrinsics.fy > 0.0f, "Depth frame intrinsics must have positive focal lengths");
  Pipeline& p = pipeline->impl;
  Pyramid& pyr = pyramid->impl;
  Tracker& t = tracker->impl;
  cudaStream_t s = p.stream;
  const bool size_changed = pyr.width != width || pyr.height != height ||
                            std::memcmp(&pyr.intrinsics, &intrinsics, sizeof(intrinsics)) != 0;
  if (p.graph_pyramid != pyramid || p.graph_tracker != tracker || size_changed) {
    check(cudaStreamSynchronize(s), "graph invalidation");
    p.clear_graphs();
    p.graph_pyramid = pyramid;
    p.graph_tracker = tracker;
  }
  pyr.prepare(width, height, intrinsics);
  const size_t n = static_cast<size_t>(width) * height;
  if (p.pixel_table.count != n) p.pixel_table.resize(n);
  if (p.frame_color.count != n) p.frame_color.resize(n);
  p.result_staging.resize(1);
  Pipeline::GraphKey key{width, height, 0, 0, 0, 0, first_frame ? 1u : 0u, has_color ? 1u : 0u, fork ? 1u : 0u,
                         cooperative && !p.concurrent ? 1u : 0u};
  uint32_t* its[4] = {&key.it0, &key.it1, &key.it2, &key.it3};
  for (uint32_t l = 0; l < 4; ++l) *its[l] = (iterations != nullptr && l < pyr.level_count) ? iterations[l] : 0u;
  if (iterations == nullptr) {
    // AppOptions::icp_iterations_for_level (app_options.cpp:147-158)
    key.it0 = 10;
    key.it1 = 5;
    key.it2 = key.it3 = 4;
  }
  auto it = p.graphs.find(key);
  if (it != p.graphs.end()) return it->second;
  // Size every buffer the graph touches before capture.
  for (uint32_t level = 0; level < pyr.level_count; ++level) p.maps_for(width >> level, height >> level);
  prepare_blocks(p, width, height, s);
  if (fork && p.side_stream == nullptr) {
    check(cudaStreamCreateWithFlags(&p.side_stream, cudaStreamNonBlocking), "side stream");
    check(cudaEventCreateWithFlags(&p.fork_event, cudaEventDisableTiming), "graph event");
    check(cudaEventCreateWithFlags(&p.pyramid_event, cudaEventDisableTiming), "graph event");
    check(cudaEventCreateWithFlags(&p.inputs_event, cudaEventDisableTiming), "graph event");
  }
  check(cudaStreamSynchronize(s), "pre-capture sync");
  cudaGraph_t graph = nullptr;
  check(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture");
  try {
    record_frame(p, pyr, t, key, has_color, s);
  } catch (...) {
    cudaStreamEndCapture(s, &graph);
    if (graph) cudaGraphDestroy(graph);
    throw;
  }
  check(cudaStreamEndCapture(s, &graph), "end capture");
  Pipeline::FrameGraph fg;
  fg.graph = graph;
  size_t nodes = 0;
  cudaError_t e = cudaGraphGetNodes(graph, nullptr, &nodes);
  if (e == cudaSuccess && nodes > 0) {
    std::vector<cudaGraphNode_t> list(nodes);
    e = cudaGraphGetNodes(graph, list.data(), &nodes);
    for (size_t i = 0; e == cudaSuccess && i < nodes; ++i) {
      cudaGraphNodeType type;
      e = cudaGraphNodeGetType(list[i], &type);
      if (e == cudaSuccess && type == cudaGraphNodeTypeKernel) ++fg.kernels;
    }
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&fg.exec, graph, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(graph);
    check(e, "graph instantiate");
  }
  return p.graphs.emplace(key, fg).first->second;
}

// Page-locked host memory (cudaHostAlloc, cudaHostRegister, a framework's
// pinned allocator) that a copy engine can read directly.
bool page_locked(const void* ptr) {
  cudaPointerAttributes attr;
  if (cudaPointerGetAttributes(&attr, ptr) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  return attr.type == cudaMemoryTypeHost;
}

// The frame's inputs into the graph's fixed buffers, on stream `s`.  Host
// buffers go through pinned staging so the copy is a true async DMA and the
// caller may reuse its buffer on return.  When the caller waits for the frame
// before returning (`caller_waits`, kf_frame_process), page-locked inputs are
// copied straight from the caller's buffers instead: no staging copy on the
// host.
void stage_inputs(Pipeline& p, Pyramid& pyr, const uint16_t* depth, const uint32_t* color, size_t n,
                  int32_t memory, cudaStream_t s, bool caller_waits = false) {
  if (memory == KF_MEMORY_DEVICE) {
    check(cudaMemcpyAsync(pyr.raw.ptr, depth, n * sizeof(uint16_t), cudaMemcpyDeviceToDevice, s), "depth copy");
    if (color) check(cudaMemcpyAsync(p.frame_color.ptr, color, n * 4, cudaMemcpyDeviceToDevice, s), "color copy");
    return;
  }
  if (!caller_waits) {
    // Frames in flight: the depth goes up on the pipeline's copy stream into
    // one of two device buffers, in turn, while the frames before it run;
    // the frame stream then only moves it into the graph's buffer on the
    // device.  A turn's buffers are reused once its previous frame's copy
    // into the graph's buffer is done.
    const int b = p.upload_turn;
    p.upload_turn ^= 1;
    if (p.copy_stream == nullptr) {
      check(cudaStreamCreateWithFlags(&p.copy_stream, cudaStreamNonBlocking), "copy stream");
      for (int i = 0; i < 2; ++i) {
        check(cudaEventCreateWithFlags(&p.uploaded[i], cudaEventDisableTiming), "upload event");
        check(cudaEventCreateWithFlags(&p.consumed[i], cudaEventDisableTiming), "upload event");
      }
    }
    check(cudaEventSynchronize(p.consumed[b]), "upload buffer reuse");  // returns at once before first use
    p.depth_pinned[b].resize(n);
    p.depth_upload[b].resize(n);
    std::memcpy(p.depth_pinned[b].ptr, depth, n * sizeof(uint16_t));
    check(cudaMemcpyAsync(p.depth_upload[b].ptr, p.depth_pinned[b].ptr, n * sizeof(uint16_t), cudaMemcpyHostToDevice,
                          p.copy_stream),
          "depth upload");
    check(cudaEventRecord(p.uploaded[b], p.copy_stream), "upload event");
    check(cudaStreamWaitEvent(s, p.uploaded[b], 0), "upload wait");
    check(cudaMemcpyAsync(pyr.raw.ptr, p.depth_upload[b].ptr, n * sizeof(uint16_t), cudaMemcpyDeviceToDevice, s),
          "depth copy");
    check(cudaEventRecord(p.consumed[b], s), "upload event");
    depth = nullptr;  // done: only the colour (if any) takes the staged path below
  }
  const bool direct_depth = depth == nullptr || (caller_waits && page_locked(depth));
  const bool direct_color = color != nullptr && caller_waits && page_locked(color);
  const bool staged = !direct_depth || (color != nullptr && !direct_color);
  // wait for the last upload from the staging before overwriting it (not for
  // the frames after it: the host fills the staging while they run)
  if (staged && p.staging_done != nullptr) check(cudaEventSynchronize(p.staging_done), "staging reuse");
  if (depth != nullptr) {
    const void* depth_src = depth;
    if (!direct_depth) {
      p.depth_staging.resize(n);
      std::memcpy(p.depth_staging.ptr, depth, n * sizeof(uint16_t));
      depth_src = p.depth_staging.ptr;
    }
    check(cudaMemcpyAsync(pyr.raw.ptr, depth_src, n * sizeof(uint16_t), cudaMemcpyHostToDevice, s), "depth upload");
  }
  if (color) {
    const void* color_src = color;
    if (!direct_color) {
      p.color_staging.resize(n);
      std::memcpy(p.color_staging.ptr, color, n * 4);
      color_src = p.color_staging.ptr;
    }
    check(cudaMemcpyAsync(p.frame_color.ptr, color_src, n * 4, cudaMemcpyHostToDevice, s), "color upload");
  }
  if (staged) {
    if (p.staging_done == nullptr) {
      check(cudaEventCreateWithFlags(&p.staging_done, cudaEventDisableTiming), "staging event");
    }
    check(cudaEventRecord(p.staging_done, s), "staging event");
  }
}

void enqueue(kf_pipeline* pipeline, kf_pyramid* pyramid, kf_tracker* tracker, const uint16_t* depth,
             const uint32_t* color, uint32_t width, uint32_t height, kf_intrinsics intrinsics, int32_t memory,
             const uint32_t* iterations, int32_t first_frame, bool caller_waits = false) {
  require(depth != nullptr, "kf_frame_enqueue: null argument");
  Pipeline::FrameGraph& fg = frame_graph_for(pipeline, pyramid, tracker, width, height, intrinsics, iterations,
                                             first_frame, color != nullptr);
  Pipeline& p = pipeline->impl;
  stage_inputs(p, pyramid->impl, depth, color, static_cast<size_t>(width) * height, memory, p.stream, caller_waits);
  check(cudaGraphLaunch(fg.exec, p.stream), "frame graph launch");
  p.last_frame_kernels = fg.kernels;
}

// `device` is the tracker state the frame ran on: a grid barrier that gave
// up during the frame is cleared there and reported as an error.
void fill_result(const IcpState& st, int first, kf_frame_result* r, IcpState* device, cudaStream_t s) {
  if (device != nullptr) check_icp_barrier(st, device, s);
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) r->camera_to_world.r[i * 3 + j] = static_cast<float>(st.pose[i * 4 + j]);
    r->camera_to_world.t[i] = static_cast<float>(st.pose[i * 4 + 3]);
  }
  r->tracked = st.failed ? 0 : 1;
  std::memcpy(r->world_to_camera.r, st.world_to_camera, 9 * sizeof(float));
  std::memcpy(r->world_to_camera.t, st.world_to_camera + 9, 3 * sizeof(float));
  for (int l = 0; l < 4; ++l) {
    r->status[l] = first ? KF_ICP_NOT_RUN : st.level_status[l];
    r->iterations[l] = first ? 0 : st.level_iterations[l];
    r->correspondences[l] = first ? 0 : st.level_correspondences[l];
  }
}

// A set of independent sequences stepped together: every member's frame
// graph becomes a child node of one parent graph, so one launch runs all of
// them concurrently (no dependencies between the branches).
struct BatchGraph {
  cudaGraphExec_t exec = nullptr;
  uint32_t kernels = 0;
};

}  // namespace
}  // namespace kf

struct kf_batch {
  std::vector<kf_pipeline*> pipelines;
  std::vector<kf_pyramid*> pyramids;
  std::vector<kf_tracker*> trackers;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  std::vector<cudaEvent_t> member_ready;
  std::map<std::vector<uint64_t>, kf::BatchGraph> graphs;
  uint32_t last_kernels = 0;
  ~kf_batch() {
    if (stream) cudaStreamSynchronize(stream);
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second.exec);
    for (cudaEvent_t e : member_ready) cudaEventDestroy(e);
    if (done) cudaEventDestroy(done);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace kf {
namespace {

void batch_step(kf_batch* b, const uint16_t* const* depths, uint32_t width, uint32_t height,
                const kf_intrinsics* intrinsics, const uint32_t* iterations, const uint8_t* first, int32_t memory) {
  require(b != nullptr && depths != nullptr && intrinsics != nullptr, "kf_batch_step: null argument");
  const size_t count = b->pipelines.size();
  std::vector<Pipeline::FrameGraph*> graphs(count, nullptr);
  std::vector<uint64_t> key(2 * count, 0);
  for (size_t i = 0; i < count; ++i) {
    if (depths[i] == nullptr) continue;  // this member sits out the step
    // one branch per member: the members already fill the GPU side by side
    graphs[i] = &frame_graph_for(b->pipelines[i], b->pyramids[i], b->trackers[i], width, height, intrinsics[i],
                                 iterations, first != nullptr && first[i] != 0, false, false, false);
    key[2 * i] = reinterpret_cast<uint64_t>(graphs[i]->graph);
    key[2 * i + 1] = b->pipelines[i]->impl.graph_epoch;
  }
  // the batch stream runs after each member's earlier work
  for (size_t i = 0; i < count; ++i) {
    if (!graphs[i]) continue;
    check(cudaEventRecord(b->member_ready[i], b->pipelines[i]->impl.stream), "batch order");
    check(cudaStreamWaitEvent(b->stream, b->member_ready[i], 0), "batch order");
  }
  for (size_t i = 0; i < count; ++i) {
    if (!graphs[i]) continue;
    stage_inputs(b->pipelines[i]->impl, b->pyramids[i]->impl, depths[i], nullptr,
                 static_cast<size_t>(width) * height, memory, b->stream);
  }
  auto it = b->graphs.find(key);
  if (it == b->graphs.end()) {
    cudaGraph_t parent = nullptr;
    check(cudaGraphCreate(&parent, 0), "batch graph");
    BatchGraph bg;
    cudaError_t e = cudaSuccess;
    for (size_t i = 0; i < count && e == cudaSuccess; ++i) {
      if (!graphs[i]) continue;
      cudaGraphNode_t node;
      e = cudaGraphAddChildGraphNode(&node, parent, nullptr, 0, graphs[i]->graph);
      bg.kernels += graphs[i]->kernels;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&bg.exec, parent, 0);
    cudaGraphDestroy(parent);
    check(e, "batch graph instantiate");
    it = b->graphs.emplace(key, bg).first;
  }
  check(cudaGraphLaunch(it->second.exec, b->stream), "batch graph launch");
  b->last_kernels = it->second.kernels;
  // later work of each member runs after the step
  check(cudaEventRecord(b->done, b->stream), "batch order");
  for (size_t i = 0; i < count; ++i) {
    if (!graphs[i]) continue;
    check(cudaStreamWaitEvent(b->pipelines[i]->impl.stream, b->done, 0), "batch order");
    b->pipelines[i]->impl.last_frame_kernels = graphs[i]->kernels;
  }
}

}  // namespace
}  // namespace kf

using namespace kf;

extern "C" {

kf_status kf_batch_create(kf_pipeline* const* pipelines, kf_pyramid* const* pyramids, kf_tracker* const* trackers,
                          uint32_t count, kf_batch** out) {
  return guarded([&] {
    require(pipelines != nullptr && pyramids != nullptr && trackers != nullptr && out != nullptr && count > 0,
            "kf_batch_create: null argument");
    auto* b = new kf_batch();
    try {
      for (uint32_t i = 0; i < count; ++i) {
        require(pipelines[i] && pyramids[i] && trackers[i], "kf_batch_create: null member");
        for (uint32_t j = 0; j < i; ++j) {
          require(pipelines[j] != pipelines[i] && pyramids[j] != pyramids[i] && trackers[j] != trackers[i],
                  "kf_batch_create: members must not share a pipeline, pyramid or tracker");
        }
        b->pipelines.push_back(pipelines[i]);
        b->pyramids.push_back(pyramids[i]);
        b->trackers.push_back(trackers[i]);
        cudaEvent_t e;
        check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "batch event");
        b->member_ready.push_back(e);
      }
      check(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "batch stream");
      check(cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming), "batch event");
    } catch (...) {
      delete b;
      throw;
    }
    *out = b;
  });
}

kf_status kf_batch_destroy(kf_batch* batch) {
  return guarded([&] { delete batch; });
}

kf_status kf_batch_step(kf_batch* batch, const uint16_t* const* depths, uint32_t width, uint32_t height,
                        const kf_intrinsics* intrinsics, const uint32_t* iterations_per_level,
                        const uint8_t* first_frame, int32_t memory) {
  return guarded(
      [&] { batch_step(batch, depths, width, height, intrinsics, iterations_per_level, first_frame, memory); });
}

kf_status kf_batch_stream(kf_batch* batch, void** stream) {
  return guarded([&] {
    require(batch != nullptr && stream != nullptr, "kf_batch_stream: null argument");
    *stream = batch->stream;
  });
}

kf_status kf_batch_kernel_count(kf_batch* batch, uint32_t* kernels) {
  return guarded([&] {
    require(batch != nullptr && kernels != nullptr, "kf_batch_kernel_count: null argument");
    *kernels = batch->last_kernels;
  });
}

kf_status kf_frame_kernel_count(kf_pipeline* pipeline, uint32_t* kernels) {
  return guarded([&] {
    require(pipeline != nullptr && kernels != nullptr, "kf_frame_kernel_count: null argument");
    *kernels = pipeline->impl.last_frame_kernels;
  });
}

kf_status kf_frame_set_pose(kf_pipeline* pipeline, kf_tracker* tracker, const kf_rigid* pose) {
  return guarded([&] {
    require(pipeline != nullptr && tracker != nullptr && pose != nullptr, "kf_frame_set_pose: null argument");
    launch_icp_set_pose(tracker->impl.state.ptr, *pose, 1, pipeline->impl.stream);
  });
}

kf_status kf_frame_enqueue(kf_pipeline* pipeline, kf_pyramid* pyramid, kf_tracker* tracker, const uint16_t* depth,
                           const uint32_t* color, uint32_t width, uint32_t height, kf_intrinsics intrinsics,
                           int32_t memory, const uint32_t* iterations_per_level, int32_t first_frame) {
  return guarded([&] {
    enqueue(pipeline, pyramid, tracker, depth, color, width, height, intrinsics, memory, iterations_per_level,
            first_frame);
  });
}

kf_status kf_frame_submit(kf_pipeline* pipeline, kf_pyramid* pyramid, kf_tracker* tracker, const uint16_t* depth,
                          const uint32_t* color, uint32_t width, uint32_t height, kf_intrinsics intrinsics,
                          int32_t memory, const uint32_t* iterations_per_level, int32_t first_frame) {
  return guarded([&] {
    require(pipeline != nullptr && tracker != nullptr, "kf_frame_submit: null argument");
    Pipeline& p = pipeline->impl;
    require(p.results_pushed - p.results_popped < static_cast<uint64_t>(Pipeline::kResultSlots),
            "kf_frame_submit: eight results are waiting; read one with kf_frame_result_next first");
    enqueue(pipeline, pyramid, tracker, depth, color, width, height, intrinsics, memory, iterations_per_level,
            first_frame);
    // the frame's result into its own slot, after the frame on the stream
    p.result_ring.resize(Pipeline::kResultSlots);
    const int slot = static_cast<int>(p.results_pushed % Pipeline::kResultSlots);
    if (p.result_ready[slot] == nullptr) {
      check(cudaEventCreateWithFlags(&p.result_ready[slot], cudaEventDisableTiming), "result event");
    }
    check(cudaMemcpyAsync(p.result_ring.ptr + slot, tracker->impl.state.ptr, sizeof(IcpState), cudaMemcpyDeviceToHost,
                          p.stream),
          "result download");
    check(cudaEventRecord(p.result_ready[slot], p.stream), "result event");
    p.result_first[slot] = first_frame ? 1 : 0;
    ++p.results_pushed;
  });
}

kf_status kf_frame_result_next(kf_pipeline* pipeline, kf_frame_result* result) {
  return guarded([&] {
    require(pipeline != nullptr && result != nullptr, "kf_frame_result_next: null argument");
    Pipeline& p = pipeline->impl;
    require(p.results_popped < p.results_pushed, "kf_frame_result_next: no submitted frame is waiting");
    const int slot = static_cast<int>(p.results_popped % Pipeline::kResultSlots);
    check(cudaEventSynchronize(p.result_ready[slot]), "frame");
    fill_result(p.result_ring.ptr[slot], p.result_first[slot], result,
                p.graph_tracker ? p.graph_tracker->impl.state.ptr : nullptr, p.stream);
    ++p.results_popped;
  });
}

kf_status kf_frame_result_fetch(kf_pipeline* pipeline, kf_frame_result* result) {
  return guarded([&] {
    require(pipeline != nullptr && result != nullptr, "kf_frame_result_fetch: null argument");
    Pipeline& p = pipeline->impl;
    check(cudaStreamSynchronize(p.stream), "frame");
    require(p.result_staging.ptr != nullptr, "kf_frame_result_fetch: no frame was processed");
    fill_result(*p.result_staging.ptr, 0, result, p.graph_tracker ? p.graph_tracker->impl.state.ptr : nullptr,
                p.stream);
  });
}

kf_status kf_frame_process(kf_pipeline* pipeline, kf_pyramid* pyramid, kf_tracker* tracker, const uint16_t* depth,
                           const uint32_t* color, uint32_t width, uint32_t height, kf_intrinsics intrinsics,
                           int32_t memory, const uint32_t* iterations_per_level, int32_t first_frame, kf_rigid* pose,
                           kf_frame_result* result) {
  return guarded([&] {
    require(pipeline && tracker && pose, "kf_frame_process: null argument");
    Pipeline& p = pipeline->impl;
    require(std::isfinite(pose->t[0]) && std::isfinite(pose->t[1]) && std::isfinite(pose->t[2]),
            "kf_frame_process: pose must be finite");
    launch_icp_set_pose(tracker->impl.state.ptr, *pose, 1, p.stream);
    enqueue(pipeline, pyramid, tracker, depth, color, width, height, intrinsics, memory, iterations_per_level,
            first_frame, true);
    check(cudaStreamSynchronize(p.stream), "frame");
    kf_frame_result local;
    fill_result(*p.result_staging.ptr, first_frame, &local, tracker->impl.state.ptr, p.stream);
    *pose = local.camera_to_world;
    if (result) *result = local;
  });
}

}  // extern "C"
