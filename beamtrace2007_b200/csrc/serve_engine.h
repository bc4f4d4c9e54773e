// The engine side of serving (bt_gpu_submit / bt_gpu_poll): what the
// request loop in serve.cpp needs from engine.cu.  Internal to the library.
#ifndef BT_SERVE_ENGINE_H
#define BT_SERVE_ENGINE_H

#include <stdint.h>

#include <shared_mutex>

#include "bt_gpu.h"

namespace btserve {

// One soft-shadow request inside a streaming run: outputs are host buffers
// (W*H each, any may be NULL), triangle ids the scene's own.
struct StreamJob {
  bt_camera cam;
  bt_area_light light;
  bt_soft_opts opts;
  int32_t scene;
  int32_t* tri;
  float* vis;
  float* E;
  float* Eu;
};

// Where a streaming run takes its jobs from and hands them back.
class SoftFeed {
 public:
  virtual ~SoftFeed() = default;
  // The next job to fold into the run, if one waits that fits in `pixels`
  // pixels and `roots` roots (a soft job of W x H pixels takes
  // ceil(W/8)*8 * ceil(H/4)*4 roots).
  virtual bool next(StreamJob& job, uint64_t& tag, int64_t pixels, int64_t roots) = 0;
  // A job's outputs are in its host buffers (status BT_OK), or it failed.
  virtual void finished(uint64_t tag, int status, const char* error) = 0;
};

// Lanes: contexts that view `parent`'s scene pool and own a stream, queues
// of `capacity` records (0: the parent's), root arrays and a pixel arena
// for `pixels` pixels in up to `jobs` jobs per run.
int laneCreate(bt_gpu_ctx* parent, int64_t capacity, int64_t pixels, int jobs, bt_gpu_ctx** out);
// Persistent CTAs per SM of a lane's kernels (bt_gpu_config.blocks_per_sm).
void laneBlocksPerSm(bt_gpu_ctx* lane, int blocks);
void laneDestroy(bt_gpu_ctx* lane);
// Takes the parent's current scene pool (call with the parent's scene lock held).
void laneView(bt_gpu_ctx* lane);

// One streaming soft-shadow run on a soft lane: takes jobs from `feed` while
// the run is younger than fold_ms, hands each back as soon as its roots are
// done.  Returns when every job it took is handed back.
int laneSoftRun(bt_gpu_ctx* lane, SoftFeed& feed, double fold_ms, bt_run_info* info);

// A primary-id image or a point-shadow mask of pool scene `scene` into host
// buffers (tri may be NULL for a mask), on the lane's stream.
int laneVisibility(bt_gpu_ctx* lane, int kind, int32_t scene, const bt_camera& cam, int32_t cull, int32_t tile,
                   const float* light, int32_t* tri, uint8_t* mask, bt_run_info* info);

// Bookkeeping for admission and the pool.
int64_t sceneBytes(const bt_gpu_ctx* c);        // the resident scene pool
int64_t laneBytes(const bt_gpu_ctx* lane);      // a lane's engine buffers as allocated
int64_t laneHighWater(const bt_gpu_ctx* lane);  // sub-beam queue bytes the lane has needed so far
int sceneCount(bt_gpu_ctx* c);
int deviceOf(const bt_gpu_ctx* c);
void useDevice(const bt_gpu_ctx* c);  // makes the context's device current on the calling thread
int64_t sceneTris(bt_gpu_ctx* c, int32_t scene);
std::shared_mutex& sceneLock(bt_gpu_ctx* c);
void*& servingState(bt_gpu_ctx* c);
const char* lastError();

// serve.cpp: ends the serving threads of `c` (bt_gpu_destroy calls it).
void stop(bt_gpu_ctx* c);

}  // namespace btserve

#endif  // BT_SERVE_ENGINE_H
