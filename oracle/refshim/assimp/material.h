// Stand-in for assimp's material header (test infrastructure): the reference's
// CMaterial declares a constructor from an aiMaterial, which nothing here calls.
#ifndef R2_REFSHIM_ASSIMP_MATERIAL_H
#define R2_REFSHIM_ASSIMP_MATERIAL_H
struct aiMaterial;
#endif
