// LOD loop of the filter with file outputs (see filter_run.cu).
#pragma once
#include <string>
#include <vector>

#include "filter_host.h"

namespace r2 {

struct FilterRunResult {
  std::vector<std::string> paths;  // per LOD: <root>/<model>/filtered_mesh_<vs> (without extension)
  double voxels = 0.0, activeVoxels = 0.0, kernelMs = 0.0;
};

FilterRunResult run_filter_lods(FilterScene& scene, const r2_filter_params& p, V3 orientation,
                                const std::string& outRoot, const std::string& model, cudaStream_t s);

}  // namespace r2
