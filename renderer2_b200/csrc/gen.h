// Seeded synthetic scene inputs (see gen.cpp).
#pragma once
#include <stdint.h>

#include <vector>

namespace r2 {

double value_noise(double x, double y, double z, uint32_t seed);
void smooth_normals(const std::vector<float>& pos, const std::vector<uint32_t>& idx, std::vector<float>* nrm);
void gen_icosphere(uint32_t subdiv, float amplitude, uint32_t seed, std::vector<float>* pos,
                   std::vector<uint32_t>* idx, std::vector<float>* nrm);
void gen_foliage(uint32_t nQuads, uint32_t nBranches, float clustered, uint32_t seed, std::vector<float>* pos,
                 std::vector<uint32_t>* idx, std::vector<float>* nrm);

}  // namespace r2
