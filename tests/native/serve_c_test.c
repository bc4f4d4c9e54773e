/* A C host of the serving entry points (include/bt_gpu.h): builds the plant
 * scene from a config, submits three mixed requests -- soft shadows,
 * primary ids, a point-shadow mask -- polls until all are handed back, and
 * checks each against the synchronous call for the same request alone
 * (bitwise).  Prints one line per request; exit status 0 = all equal.
 *
 *   serve_c_test [W]            (needs a CUDA device) */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "bt_gpu.h"

#define CHECK(x)                                                               \
  do {                                                                         \
    int rc_ = (x);                                                             \
    if (rc_ != BT_OK) {                                                        \
      fprintf(stderr, "%s: %d %s\n", #x, rc_, bt_gpu_last_error());            \
      return 2;                                                                \
    }                                                                          \
  } while (0)

static int same(const void* a, const void* b, size_t n, const char* what) {
  const int eq = memcmp(a, b, n) == 0;
  printf("%-22s %s\n", what, eq ? "equal" : "DIFFERENT");
  return eq;
}

int main(int argc, char** argv) {
  const int W = argc > 1 ? atoi(argv[1]) : 96, H = W * 3 / 4;
  const char* cfg =
      "name plant\nmesh procedural plant\nup 0 1 0\nview 2.6 1.7 3.4  0 0.55 0  45\n"
      "point_light 1.0 3.0 0.8\narea_light 0.9 2.8 0.7  0.4 0 0  0 0 0.4\n";
  bt_scene_file* sf = NULL;
  CHECK(bt_scene_parse_config(cfg, &sf));
  bt_scene_file_info fi;
  bt_scene_file_info_get(sf, &fi);
  float* pos = malloc(sizeof(float) * 3 * fi.num_verts);
  uint32_t* tris = malloc(sizeof(uint32_t) * 3 * fi.num_tris);
  float* views = malloc(sizeof(float) * 7 * fi.num_views);
  bt_scene_file_arrays(sf, pos, tris, NULL, NULL, views);
  /* finalise, kd-tree, context */
  uint32_t* ftris = malloc(sizeof(uint32_t) * 3 * fi.num_tris);
  float* nrm = malloc(sizeof(float) * 3 * fi.num_tris);
  float* area = malloc(sizeof(float) * fi.num_tris);
  bt_scene_desc sd;
  const int64_t nt = bt_scene_finalize(pos, fi.num_verts, tris, fi.num_tris, ftris, nrm, area, sd.bounds);
  if (nt <= 0) return 2;
  sd.pos = pos;
  sd.num_verts = fi.num_verts;
  sd.tris = ftris;
  sd.tri_normals = nrm;
  sd.num_tris = nt;
  bt_kd_params kp;
  bt_kd_params_default(&kp);
  bt_kd_tree* tree = NULL;
  CHECK(bt_kd_build(pos, ftris, area, nt, sd.bounds, &kp, &tree));
  bt_kd_desc kd;
  bt_kd_view(tree, &kd);
  bt_gpu_ctx* ctx = NULL;
  CHECK(bt_gpu_create(&sd, &kd, NULL, &ctx));
  bt_camera cam;
  bt_camera_make(views, views + 3, views[6], fi.up, W, H, &cam);
  bt_area_light L;
  memcpy(L.c, fi.light_c, sizeof L.c);
  memcpy(L.U, fi.light_u, sizeof L.U);
  memcpy(L.V, fi.light_v, sizeof L.V);
  bt_soft_opts opts = {1, 0.0f};
  const size_t n = (size_t)W * H;

  /* the three requests, submitted back to back */
  int32_t* s_tri = calloc(n, 4);
  float *s_vis = calloc(n, 4), *s_E = calloc(n, 4), *s_Eu = calloc(n, 4);
  int32_t* p_tri = calloc(n, 4);
  uint8_t* m_mask = calloc(n, 1);
  bt_request rq[3];
  memset(rq, 0, sizeof rq);
  for (int k = 0; k < 3; ++k) {
    rq[k].scene = 0;
    rq[k].cam = cam;
    rq[k].tile = 16;
    rq[k].user = 100 + k;
  }
  rq[0].kind = BT_REQ_SOFT;
  rq[0].light = L;
  rq[0].opts = opts;
  rq[0].tri = s_tri;
  rq[0].vis = s_vis;
  rq[0].E = s_E;
  rq[0].Eu = s_Eu;
  rq[1].kind = BT_REQ_PRIMARY_IDS;
  rq[1].tri = p_tri;
  rq[2].kind = BT_REQ_POINT_MASK;
  memcpy(rq[2].point_light, fi.point_light, sizeof rq[2].point_light);
  rq[2].mask = m_mask;
  uint64_t tickets[3];
  for (int k = 0; k < 3; ++k) CHECK(bt_gpu_submit(ctx, &rq[k], &tickets[k]));
  int got = 0, ok = 1;
  while (got < 3) {
    bt_completion c[4];
    int32_t cnt = 0;
    CHECK(bt_gpu_poll(ctx, c, 4, &cnt, 1000));
    for (int i = 0; i < cnt; ++i) {
      printf("ticket %llu (user %llu, kind %d): status %d, %.2f ms\n", (unsigned long long)c[i].ticket,
             (unsigned long long)c[i].user, c[i].kind, c[i].status, c[i].ms_total);
      ok &= c[i].status == BT_OK && c[i].user == 100 + (uint64_t)c[i].kind;
    }
    got += cnt;
  }
  bt_serve_stats st;
  CHECK(bt_gpu_serve_stats(ctx, &st));
  printf("submitted %lld completed %lld soft runs %lld\n", (long long)st.submitted, (long long)st.completed,
         (long long)st.soft_runs);
  ok &= st.submitted == 3 && st.completed == 3;

  /* the same requests alone, through the synchronous entry points */
  int32_t* a_tri = calloc(n, 4);
  float *a_vis = calloc(n, 4), *a_E = calloc(n, 4), *a_Eu = calloc(n, 4);
  CHECK(bt_gpu_soft(ctx, &cam, &L, &opts, a_tri, a_vis, a_E, a_Eu, NULL));
  ok &= same(s_tri, a_tri, 4 * n, "soft tri");
  ok &= same(s_vis, a_vis, 4 * n, "soft vis");
  ok &= same(s_E, a_E, 4 * n, "soft E");
  ok &= same(s_Eu, a_Eu, 4 * n, "soft Eu");
  int32_t* a_ids = calloc(n, 4);
  CHECK(bt_gpu_primary_ids(ctx, &cam, 0, 16, a_ids, NULL));
  ok &= same(p_tri, a_ids, 4 * n, "primary ids");
  uint8_t* a_mask = calloc(n, 1);
  CHECK(bt_gpu_point_mask(ctx, &cam, 0, 16, fi.point_light, NULL, a_mask, NULL));
  ok &= same(m_mask, a_mask, n, "point mask");
  int shaded = 0, shadowed = 0;
  for (size_t i = 0; i < n; ++i) {
    shaded += a_tri[i] >= 0;
    shadowed += a_mask[i] != 0;
  }
  printf("%d shaded px, %d shadowed px\n", shaded, shadowed);
  ok &= shaded > (int)(n / 8) && shadowed > 0;
  CHECK(bt_gpu_destroy(ctx));
  bt_kd_free(tree);
  bt_scene_file_free(sf);
  printf(ok ? "serve_c_test: ok\n" : "serve_c_test: FAILED\n");
  return ok ? 0 : 1;
}
