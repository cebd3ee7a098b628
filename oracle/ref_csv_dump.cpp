// TEST INFRASTRUCTURE ONLY: drives the reference's CSV reader (src/core/utils/csv.hpp) with the two configurations
// the reference reads files with, so that this project's CSV readers can be checked against it.
//
// Built by oracle/ref_build.py (build_csv_dump) with the reference's src/ directory on the include path.
//   ref_csv_dump comp <in.csv> <out.bin>  -- DEMClumpTemplate::ReadComponentFromFile (src/DEM/Structs.h:419-437):
//        io::CSVReader<4> with its default policies, header read with ignore_missing_column, columns x, y, z, r
//   ref_csv_dump xyz <in.csv> <out.bin>   -- DEMSolver::ReadClumpXyzFromCsv (src/DEM/API.h:328-347): trimmed cells,
//        empty lines skipped, header read with ignore_extra_column, columns clump_type, X, Y, Z
// out.bin: int32 row count, then per row four float32 (comp: x, y, z, r; xyz: X, Y, Z and the row's clump-type
// name length as a float), then the names (xyz only), each as int32 length + bytes.
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "core/utils/csv.hpp"

int main(int argc, char** argv) {
    if (argc != 4) return 2;
    const std::string mode = argv[1];
    std::vector<float> vals;
    std::vector<std::string> names;
    if (mode == "comp") {
        deme::io::CSVReader<4> in(argv[2]);
        in.read_header(deme::io::ignore_missing_column, "x", "y", "z", "r");
        float x = 0, y = 0, z = 0, r = 0;
        while (in.read_row(x, y, z, r)) vals.insert(vals.end(), {x, y, z, r});
    } else if (mode == "xyz") {
        deme::io::CSVReader<4, deme::io::trim_chars<' ', '\t'>, deme::io::no_quote_escape<','>,
                            deme::io::throw_on_overflow, deme::io::empty_line_comment>
            in(argv[2]);
        in.read_header(deme::io::ignore_extra_column, "clump_type", "X", "Y", "Z");
        std::string name;
        float x, y, z;
        while (in.read_row(name, x, y, z)) {
            vals.insert(vals.end(), {x, y, z, (float)name.size()});
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
