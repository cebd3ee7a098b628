// TEST INFRASTRUCTURE ONLY: drives the reference's own Wavefront OBJ parser, so that the mesh loaders of this
// project (deme_b200.scene.load_wavefront and deme::DEMMeshConnected::LoadWavefrontMesh) can be checked against it.
//
// Built by oracle/ref_build.py (build_obj_dump) with the reference's src/ directory on the include path; the parser
// itself is the header src/core/utils/WavefrontMeshLoader.hpp, used here exactly as
// DEMMeshConnected::LoadWavefrontMesh (src/DEM/MeshUtils.cpp:44-112) uses it: OBJ::LoadMesh with an empty geometry
// callback, then the flat arrays mVerts / mIndexesVerts / mNormals / mIndexesNormals read three at a time.
//
// usage: ref_obj_dump <in.obj> <out.bin>
// out.bin: int32 counts (vertices, facets, normals, facet normal triples), then the vertices (float32 x3), the facet
// vertex indices (int32 x3, 0-based as the reference stores them), the normals (float32 x3) and the facet normal
// indices (int32 x3).  Exit status 1 when the reference's loader reports a failure.
#include <strings.h>

#include <cstdint>
#include <cstdio>
#include <vector>

#include "core/utils/WavefrontMeshLoader.hpp"

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s in.obj out.bin\n", argv[0]);
        return 2;
    }
    deme::WAVEFRONT::GeometryInterface none;
    deme::WAVEFRONT::OBJ obj;
    if (obj.LoadMesh(argv[1], &none, true) == -1) return 1;
    const int32_t counts[4] = {(int32_t)(obj.mVerts.size() / 3), (int32_t)(obj.mIndexesVerts.size() / 3),
                               (int32_t)(obj.mNormals.size() / 3), (int32_t)(obj.mIndexesNormals.size() / 3)};
    std::FILE* f = std::fopen(argv[2], "wb");
    if (!f) return 2;
    std::fwrite(counts, sizeof(int32_t), 4, f);
    std::fwrite(obj.mVerts.data(), sizeof(float), 3 * (size_t)counts[0], f);
    std::fwrite(obj.mIndexesVerts.data(), sizeof(int), 3 * (size_t)counts[1], f);
    std::fwrite(obj.mNormals.data(), sizeof(float), 3 * (size_t)counts[2], f);
    std::fwrite(obj.mIndexesNormals.data(), sizeof(int), 3 * (size_t)counts[3], f);
    std::fclose(f);
    return 0;
}
