// r2 <config.json>: the pipeline of the reference's `raytracer <config.json>`
// (raytracer/main.cu:4-18 running CPipeline::run, raytracer/pipeline.cu:24-90
// without its GUI): optional filtering of the FILTER mesh into ./filtering,
// one frame, ./output.png (tonemapped, gamma-corrected) and ./output.hdr (the
// linear frame).  The reference's output.jpg is not written.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <chrono>
#include <vector>

#include "r2.h"

static int fail(r2_status s, const char* what) {
  fprintf(stderr, "r2: %s failed: %s: %s\n", what, r2_status_string(s), r2_last_error());
  return 1;
}

int main(int argc, char** argv) {
  if (argc < 2) {
    fprintf(stderr, "usage: r2 <config.json> [--spp N] [--seed S]\n");
    return 2;
  }
  r2_render_opts opts;
  memset(&opts, 0, sizeof(opts));
  for (int i = 2; i + 1 < argc; i += 2) {
    if (strcmp(argv[i], "--spp") == 0) opts.spp = (uint32_t)strtoul(argv[i + 1], nullptr, 10);
    else if (strcmp(argv[i], "--seed") == 0) opts.seed = (uint32_t)strtoul(argv[i + 1], nullptr, 10);
  }
  r2_config* cfg = nullptr;
  r2_status s = r2_config_load(argv[1], &cfg);
  if (s != R2_OK) return fail(s, "config");
  r2_config_info info;
  r2_config_info_get(cfg, &info);
  if (info.filter_active) {
    auto t0 = std::chrono::steady_clock::now();
    double st[4];
    s = r2_filter_run(cfg, "./filtering", st);
    if (s != R2_OK) return fail(s, "filtering");
    std::chrono::duration<double> d = std::chrono::steady_clock::now() - t0;
    printf("Filtering took %f s (%d LODs, %.0f voxels)\n", d.count(), (int)st[0], st[1]);
  }
  const size_t n = (size_t)info.frame_width * info.frame_height * 3;
  std::vector<float> linear(n);
  std::vector<uint8_t> bytes(n);
  auto t0 = std::chrono::steady_clock::now();
  s = r2_render(cfg, &opts, linear.data(), bytes.data());
  if (s != R2_OK) return fail(s, "render");
  std::chrono::duration<double> d = std::chrono::steady_clock::now() - t0;
  printf("Rendering took %f s\n", d.count());
  s = r2_write_jpg("./output.jpg", bytes.data(), info.frame_width, info.frame_height, 1, 100);
  if (s != R2_OK) return fail(s, "output.jpg");
  s = r2_write_png("./output.png", bytes.data(), info.frame_width, info.frame_height, 1);
  if (s != R2_OK) return fail(s, "output.png");
  // the frame's row 0 is the bottom; .hdr files start at the top
  std::vector<float> top(n);
  const size_t row = (size_t)info.frame_width * 3;
  for (uint32_t y = 0; y < info.frame_height; ++y)
    memcpy(&top[(size_t)y * row], &linear[(size_t)(info.frame_height - 1 - y) * row], row * sizeof(float));
  s = r2_write_hdr("./output.hdr", top.data(), info.frame_width, info.frame_height);
  if (s != R2_OK) return fail(s, "output.hdr");
  r2_config_free(cfg);
  return 0;
}
