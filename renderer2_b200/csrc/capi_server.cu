// C ABI of the request loop (server.h).
#include <memory>

#include "capi_util.h"
#include "server.h"

struct r2_scene;
struct r2_filter_scene;
r2::RenderScene* r2_scene_impl(r2_scene* scene);
r2::FilterScene* r2_filter_scene_impl(r2_filter_scene* scene);

struct r2_server {
  std::unique_ptr<r2::Server> impl;
};

extern "C" {

r2_status r2_server_create(uint32_t slots, uint64_t hbm_budget_bytes, r2_server** out) {
  R2_API_BEGIN
  R2_REQUIRE(out, R2_ERR_INVALID_ARGUMENT, "null argument");
  r2::require_device();
  std::unique_ptr<r2_server> s(new r2_server());
  s->impl.reset(new r2::Server(slots, hbm_budget_bytes));
  *out = s.release();
  R2_API_END
}

r2_status r2_server_destroy(r2_server* server) {
  R2_API_BEGIN
  delete server;
  R2_API_END
}

r2_status r2_server_render_bytes(r2_scene* scene, const r2_camera* camera, const r2_render_params* params,
                                 uint64_t* bytes_out) {
  R2_API_BEGIN
  R2_REQUIRE(scene && camera && params && bytes_out, R2_ERR_INVALID_ARGUMENT, "null argument");
  R2_REQUIRE(camera->width > 0 && camera->height > 0 && params->spp > 0, R2_ERR_INVALID_ARGUMENT, "empty job");
  *bytes_out = r2::Server::render_bytes(*r2_scene_impl(scene), *camera, *params);
  R2_API_END
}

r2_status r2_server_submit_render(r2_server* server, r2_scene* scene, const r2_camera* camera,
                                  const r2_render_params* params, float* rgb_out, uint64_t* job_id) {
  R2_API_BEGIN
  R2_REQUIRE(server && scene && camera && params && rgb_out && job_id, R2_ERR_INVALID_ARGUMENT, "null argument");
  R2_REQUIRE((params->flags & ~R2_RENDER_BRICK_GRID) == 0, R2_ERR_INVALID_ARGUMENT, "unknown render flags");
  std::unique_ptr<r2::ServerJob> j(new r2::ServerJob());
  j->kind = 0;
  j->scene = r2_scene_impl(scene);
  j->cam = *camera;
  j->rp = *params;
  j->rgbOut = rgb_out;
  *job_id = server->impl->submit(std::move(j));
  R2_API_END
}

r2_status r2_server_submit_filter(r2_server* server, r2_filter_scene* scene, const r2_filter_grid* grid,
                                  const r2_filter_params* params, uint32_t lod, r2_voxel* out, uint64_t* job_id) {
  R2_API_BEGIN
  R2_REQUIRE(server && scene && grid && params && out && job_id, R2_ERR_INVALID_ARGUMENT, "null argument");
  std::unique_ptr<r2::ServerJob> j(new r2::ServerJob());
  j->kind = 1;
  j->fscene = r2_filter_scene_impl(scene);
  j->grid = *grid;
  j->fp = *params;
  j->lod = lod;
  j->voxOut = out;
  *job_id = server->impl->submit(std::move(j));
  R2_API_END
}

r2_status r2_server_wait(r2_server* server, uint64_t job_id, double timeout_s, double* times_out) {
  R2_API_BEGIN
  R2_REQUIRE(server, R2_ERR_INVALID_ARGUMENT, "null argument");
  r2::ServerJob j;
  if (!server->impl->wait(job_id, timeout_s, &j)) return R2_ERR_PENDING;
  if (times_out) {
    times_out[0] = j.tSubmit;
    times_out[1] = j.tStart;
    times_out[2] = j.tEnd;
  }
  if (j.status != R2_OK) {
    r2::set_last_error(j.error);
    return j.status;
  }
  R2_API_END
}

r2_status r2_server_stats(r2_server* server, double* stats_out) {
  R2_API_BEGIN
  R2_REQUIRE(server && stats_out, R2_ERR_INVALID_ARGUMENT, "null argument");
  server->impl->stats(stats_out);
  R2_API_END
}

}  // extern "C"
