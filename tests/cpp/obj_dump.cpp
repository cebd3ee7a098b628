// Reads a Wavefront OBJ file with deme::DEMMeshConnected (include/deme_solver.hpp) and writes what it holds, so that
// tests/test_mesh_loader.py can compare it with the Python front end and with the reference's own parser.
//
// usage: obj_dump <in.obj> <out.bin> [<written.obj>]
// out.bin: int32 counts (vertices, facets, normals, facet normal triples), the vertices (float32 x3), the facet
// vertex indices (int32 x3), the normals (float32 x3), the facet normal indices (int32 x3), then an int32 flag and,
// when it is 1, every facet's nodes after UseNormals (float32 x9 per facet), then the same four counts and arrays
// for the merge of the mesh with itself.  <written.obj>: WriteWavefront of {mesh, mesh without normals}.
#include <cstdint>
#include <cstdio>
#include <vector>

#include "deme_solver.hpp"

using deme::DEMMeshConnected;

static void put_mesh(std::FILE* f, const DEMMeshConnected& m) {
    const int32_t counts[4] = {(int32_t)m.vertices.size(), (int32_t)m.face_v_indices.size(),
                               (int32_t)m.normals.size(), (int32_t)m.face_n_indices.size()};
    std::fwrite(counts, sizeof(int32_t), 4, f);
    std::fwrite(m.vertices.data(), sizeof(float3), m.vertices.size(), f);
    std::fwrite(m.face_v_indices.data(), sizeof(int3), m.face_v_indices.size(), f);
    std::fwrite(m.normals.data(), sizeof(float3), m.normals.size(), f);
    std::fwrite(m.face_n_indices.data(), sizeof(int3), m.face_n_indices.size(), f);
}

int main(int argc, char** argv) {
    if (argc != 3 && argc != 4) {
        std::fprintf(stderr, "usage: %s in.obj out.bin [written.obj]\n", argv[0]);
        return 2;
    }
    DEMMeshConnected m;
    if (!m.LoadWavefrontMesh(argv[1])) return 1;
    std::FILE* f = std::fopen(argv[2], "wb");
    if (!f) return 2;
    put_mesh(f, m);
    const int32_t oriented = m.face_n_indices.size() == m.GetNumTriangles() && m.GetNumTriangles() > 0;
    std::fwrite(&oriented, sizeof(int32_t), 1, f);
    if (oriented) {
        m.UseNormals();
        for (size_t i = 0; i < m.GetNumTriangles(); i++) {
            const std::array<float3, 3> t = m.FacetNodes(i);
            std::fwrite(t.data(), sizeof(float3), 3, f);
        }
        m.UseNormals(false);
    }
    std::vector<DEMMeshConnected> two{m, m};
    put_mesh(f, DEMMeshConnected::Merge(two));
    std::fclose(f);
    if (argc == 4) {
        DEMMeshConnected bare = m;
        bare.normals.clear();
        bare.face_n_indices.clear();
        std::vector<DEMMeshConnected> pair{m, bare};
        DEMMeshConnected::WriteWavefront(argv[3], pair);
    }
    return 0;
}
