// Reads a CSV file with the C++ facade's readers (include/deme_solver.hpp) and writes what they return in the
// format of oracle/ref_csv_dump.cpp, so that tests/test_csv_numbers.py can compare them with the reference's reader.
//   csv_dump comp <in.csv> <out.bin>  -- DEMClumpTemplate::ReadComponentFromFile (columns x, y, z, r)
//   csv_dump xyz <in.csv> <out.bin>   -- DEMSolver::ReadClumpXyzFromCsv (columns clump_type, X, Y, Z), the names
//        in sorted order, file order within a name
// out.bin: int32 row count, then per row four float32, then (xyz) each row's name as int32 length + bytes.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "deme_solver.hpp"

int main(int argc, char** argv) {
    if (argc != 4) return 2;
    const std::string mode = argv[1];
    std::vector<float> vals;
    std::vector<std::string> names;
    if (mode == "comp") {
        deme::DEMClumpTemplate t;
        if (t.ReadComponentFromFile(argv[2])) return 1;
        for (size_t i = 0; i < t.radii.size(); i++)
            vals.insert(vals.end(), {t.relPos[i].x, t.relPos[i].y, t.relPos[i].z, t.radii[i]});
    } else if (mode == "xyz") {
        const auto m = deme::DEMSolver::ReadClumpXyzFromCsv(argv[2]);
        std::vector<std::string> order;
        for (const auto& kv : m) order.push_back(kv.first);
        std::sort(order.begin(), order.end());
        for (const auto& name : order)
            for (const float3& p : m.at(name)) {
                vals.insert(vals.end(), {p.x, p.y, p.z, (float)name.size()});
                names.push_back(name);
            }
    } else {
        return 2;
    }
    std::FILE* f = std::fopen(argv[3], "wb");
    if (!f) return 2;
    const int32_t n = (int32_t)(vals.size() / 4);
    std::fwrite(&n, sizeof(n), 1, f);
    std::fwrite(vals.data(), sizeof(float), vals.size(), f);
    for (const auto& s : names) {
        const int32_t l = (int32_t)s.size();
        std::fwrite(&l, sizeof(l), 1, f);
        std::fwrite(s.data(), 1, s.size(), f);
    }
    std::fclose(f);
    return 0;
}
