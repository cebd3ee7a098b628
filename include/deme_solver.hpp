/* deme_solver.hpp -- C++ DEMSolver facade over the C ABI of deme_b200.h (header-only, C++17).
 *
 * Keeps the scene-building and stepping API of deme::DEMSolver (src/DEM/API.h:44-887): LoadMaterial,
 * LoadClumpType / LoadSphereType, AddClumps (DEMClumpBatch setters), AddExternalObject / AddBCPlane
 * (DEMExternObj::AddPlane, plus AddCylinder / AddCone), AddWavefrontMeshObject (DEMMeshConnected), the family controls, DefineContactForceModel with
 * SetPerContactWildcards, the world and time-stepping setters, Initialize, DoDynamics / DoDynamicsThenSync /
 * DoStepDynamics and owner-state queries.  Initialize flattens the scene exactly as the reference's host code does
 * before its JIT step (src/DEM/APIPrivate.cpp:222-369, 574-687, 903-1048; src/DEM/dT.cpp:480-640;
 * src/DEM/HostSideHelpers.hpp:328-350) and hands the flat arrays to deme_create.  The Python SceneBuilder
 * (deme_b200/scene.py) implements the same flattening; tests check that the two agree array by array.
 *
 * Prescribed motions that are plain numbers go into the per-family constant table; a family with any other string
 * (a C expression of the time t, as the reference accepts) is compiled at Initialize into the integration kernel
 * by deme_set_prescribed_motion.  Errors throw std::runtime_error with the library's message, as DEME_ERROR does.
 */
#ifndef DEME_SOLVER_HPP
#define DEME_SOLVER_HPP

#include <algorithm>
#include <array>
#include <cctype>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <memory>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include <vector_functions.h>
#include <vector_types.h>

#include "deme_b200.h"

namespace deme {

enum class TIME_INTEGRATOR { FORWARD_EULER = 0, CENTERED_DIFFERENCE = 1, EXTENDED_TAYLOR = 2 };
// src/DEM/Defines.h:104, 114: verbosity levels (accepted, no effect here) and output formats (CSV is written)
enum VERBOSITY { QUIET = 0, ERROR = 10, WARNING = 20, INFO = 30, STEP_STATS = 32, STEP_METRIC = 35, DEBUG = 40 };
enum class OUTPUT_FORMAT { CSV, BINARY, CHPF };
enum class FORCE_MODEL { HERTZIAN, HERTZIAN_FRICTIONLESS, CUSTOM };  // src/DEM/Defines.h:116

class DEMMaterial {
  public:
    explicit DEMMaterial(const std::unordered_map<std::string, float>& props, unsigned order)
        : mat_prop(props), load_order(order) {}
    std::unordered_map<std::string, float> mat_prop;
    unsigned load_order;
};

/* A CSV cell's float as the reference's CSV reader forms it (io::detail::parse_float<float>,
 * src/core/utils/csv.hpp:936-997, behind DEMClumpTemplate::ReadComponentFromFile and ReadClumpXyzFromCsv /
 * ReadClumpQuatFromCsv).  That reader is not correctly rounded: integer digits accumulate in float (x = x * 10 + d),
 * each fraction digit adds d * p with p divided by 10 per digit in float, and an exponent is applied by repeated
 * squaring of 10 or 0.1 in float; the same float operations in the same order are done here, each product stored
 * before it is added so that no compiler fuses them.  Spaces and tabs around the cell are ignored; an empty cell is
 * 0.  An exponent written with '+' is read (the reference rejects it).  Anything else throws
 * std::invalid_argument. */
inline float csv_float(const std::string& cell) {
    size_t i = cell.find_first_not_of(" \t\r"), end = cell.find_last_not_of(" \t\r");
    if (i == std::string::npos) return 0.f;
    end++;
    auto bad = [&]() { return std::invalid_argument("not a number in a CSV cell: '" + cell + "'"); };
    const bool neg = cell[i] == '-';
    if (cell[i] == '-' || cell[i] == '+') i++;
    volatile float x = 0.f;
    auto digit = [&](size_t k) { return k < end && cell[k] >= '0' && cell[k] <= '9'; };
    for (; digit(i); i++) {
        x = x * 10.f;
        x = x + (float)(cell[i] - '0');
    }
    if (i < end && (cell[i] == '.' || cell[i] == ',')) {
        i++;
        float pos = 1.f;
        for (; digit(i); i++) {
            pos = pos / 10.f;
            const volatile float term = (float)(cell[i] - '0') * pos;
            x = x + term;
        }
    }
    if (i < end && (cell[i] == 'e' || cell[i] == 'E')) {
        i++;
        bool eneg = false;
        if (i < end && (cell[i] == '-' || cell[i] == '+')) eneg = cell[i++] == '-';
        long e = 0;
        for (; i < end; i++) {
            if (!digit(i)) throw bad();
            e = std::min(e * 10 + (cell[i] - '0'), 1L << 20);
        }
        if (e != 0) {
            float base = eneg ? 0.1f : 10.f;
            while (e != 1) {
                if ((e & 1) == 0) {
                    base = base * base;
                    e >>= 1;
                } else {
                    x = x * base;
                    --e;
                }
            }
            x = x * base;
        }
    } else if (i != end) {
        throw bad();
    }
    return neg ? -x : x;
}

class DEMClumpTemplate {
  public:
    std::string m_name = "NULL";  // "%04d" of the load count unless assigned (src/DEM/APIPublic.cpp:337-341)
    void AssignName(const std::string& some_name) { m_name = some_name; }
    float mass = 0.f;
    float3 MOI{0.f, 0.f, 0.f};
    std::vector<float> radii;
    std::vector<float3> relPos;
    std::vector<std::shared_ptr<DEMMaterial>> materials;
    unsigned mark = 0;
    float volume = 0.f;  // for the "clump_volume" inspector (DEMClumpTemplate::SetVolume)
    void SetVolume(float vol) { volume = vol; }
    unsigned nComp() const { return (unsigned)radii.size(); }
    /* ReadComponentFromFile (src/DEM/Structs.h:419-437): sphere components from a CSV file with a header row;
     * the columns named x_id, y_id, z_id and r_id, in any order among others (a missing one or an empty cell reads
     * 0), are appended, the numbers formed as the reference's reader forms them (csv_float).  Lines starting with
     * '#' and blank lines are skipped, as by that reader's default comment policy.  Returns 0, or 1 if the file
     * cannot be read. */
    int ReadComponentFromFile(const std::string& filename, const std::string& x_id = "x",
                              const std::string& y_id = "y", const std::string& z_id = "z",
                              const std::string& r_id = "r") {
        std::ifstream in(filename);
        if (!in) return 1;
        auto split = [](const std::string& line) {
            std::vector<std::string> out;
            std::stringstream ss(line);
            std::string cell;
            while (std::getline(ss, cell, ',')) {
                const size_t b = cell.find_first_not_of(" \t\r"), e = cell.find_last_not_of(" \t\r");
                out.push_back(b == std::string::npos ? std::string() : cell.substr(b, e - b + 1));
            }
            return out;
        };
        std::string line;
        auto skipped = [](const std::string& l) {
            return l.find_first_not_of(" \t\r") == std::string::npos || (!l.empty() && l[0] == '#');
        };
        do {
            if (!std::getline(in, line)) return 0;
        } while (skipped(line));
        const std::vector<std::string> head = split(line);
        int col[4] = {-1, -1, -1, -1};
        const std::string* ids[4] = {&x_id, &y_id, &z_id, &r_id};
        for (int k = 0; k < 4; k++)
            for (size_t c = 0; c < head.size(); c++)
                if (head[c] == *ids[k]) col[k] = (int)c;
        while (std::getline(in, line)) {
            if (skipped(line)) continue;
            const std::vector<std::string> row = split(line);
            float v[4] = {0.f, 0.f, 0.f, 0.f};
            for (int k = 0; k < 4; k++)
                if (col[k] >= 0 && (size_t)col[k] < row.size()) v[k] = csv_float(row[col[k]]);
            relPos.push_back(float3{v[0], v[1], v[2]});
            radii.push_back(v[3]);
        }
        return 0;
    }
};

class DEMClumpBatch {
  public:
    explicit DEMClumpBatch(size_t n) : nClumps(n), vel(n, float3{0, 0, 0}), angVel(n, float3{0, 0, 0}),
                                       oriQ(n, float4{0, 0, 0, 1}), families(n, 0) {}
    size_t GetNumClumps() const { return nClumps; }
    void SetTypes(const std::vector<std::shared_ptr<DEMClumpTemplate>>& t) { check(t.size(), "SetTypes"); types = t; }
    void SetTypes(const std::shared_ptr<DEMClumpTemplate>& t) { SetTypes({nClumps, t}); }
    void SetType(const std::shared_ptr<DEMClumpTemplate>& t) { SetTypes({nClumps, t}); }
    void SetPos(const std::vector<float3>& p) { check(p.size(), "SetPos"); xyz = p; }
    void SetPos(float3 p) { SetPos(std::vector<float3>(nClumps, p)); }
    void SetVel(const std::vector<float3>& v) { check(v.size(), "SetVel"); vel = v; }
    void SetVel(float3 v) { SetVel(std::vector<float3>(nClumps, v)); }
    void SetAngVel(const std::vector<float3>& w) { check(w.size(), "SetAngVel"); angVel = w; }
    void SetAngVel(float3 w) { SetAngVel(std::vector<float3>(nClumps, w)); }
    /* quaternions as float4 with .w the scalar part (the reference's convention) */
    void SetOriQ(const std::vector<float4>& q) { check(q.size(), "SetOriQ"); oriQ = q; }
    void SetOriQ(float4 q) { SetOriQ(std::vector<float4>(nClumps, q)); }
    void SetFamilies(const std::vector<unsigned>& f) {
        check(f.size(), "SetFamilies");
        for (unsigned v : f)
            if (v > 255) throw std::runtime_error("Some clumps are instructed to have a family number larger than 255");
        families = f;
    }
    void SetFamilies(unsigned f) { SetFamilies(std::vector<unsigned>(nClumps, f)); }
    void SetFamily(unsigned f) { SetFamilies(f); }

    size_t nClumps;
    std::vector<std::shared_ptr<DEMClumpTemplate>> types;
    std::vector<float3> xyz, vel, angVel;
    std::vector<float4> oriQ;
    std::vector<unsigned> families;

  private:
    void check(size_t n, const char* what) const {
        if (n != nClumps) throw std::runtime_error(std::string(what) + ": input length does not match the batch");
    }
};

struct DEMAnalEntity {
    int type;  // DEME_ANAL_*
    std::shared_ptr<DEMMaterial> material;
    float3 pos, rot;
    float size1, size2, size3;
    int normal;  // 0 inward (default), 1 outward
};

class DEMExternObj {
  public:
    explicit DEMExternObj(unsigned order) : load_order(order) {}
    void SetFamily(unsigned code) {
        if (code > 255) throw std::runtime_error("family number is larger than the max allowance 255");
        family_code = code;
    }
    void SetMass(float m) { mass = m; }
    void SetMOI(float3 moi) { MOI = moi; }
    void SetInitPos(float3 p) { init_pos = p; }
    void AddPlane(float3 pos, float3 normal, const std::shared_ptr<DEMMaterial>& mat) {
        entities.push_back({DEME_ANAL_PLANE, mat, pos, normalize_host(normal), 0.f, 0.f, 0.f, 0});
    }
    /* AddPlate (BdrsAndObjs.h:152-170): kept with its half sizes; as in the reference (DEMHelperKernels.cu:385-387,
     * 439-441) it meets no sphere */
    void AddPlate(float3 pos, float3 normal, float xdim, float ydim, const std::shared_ptr<DEMMaterial>& mat) {
        entities.push_back({DEME_ANAL_PLATE, mat, pos, normalize_host(normal), (float)(xdim / 2.0),
                            (float)(ydim / 2.0), 0.f, 0});
    }
    /* infinite cylinder through `point` along `axis`; spheres live inside unless normal_outward */
    void AddCylinder(float3 point, float3 axis, float radius, const std::shared_ptr<DEMMaterial>& mat,
                     bool normal_outward = false) {
        entities.push_back({DEME_ANAL_CYLINDER, mat, point, normalize_host(axis), radius, 0.f, 0.f, normal_outward});
    }
    /* cone with apex `apex` opening along `axis`; the wall exists for axial distances [u_min, u_max] */
    void AddCone(float3 apex, float3 axis, float half_angle, float u_min, float u_max,
                 const std::shared_ptr<DEMMaterial>& mat, bool normal_outward = false) {
        entities.push_back({DEME_ANAL_CONE, mat, apex, normalize_host(axis), half_angle, u_min, u_max, normal_outward});
    }
    /* helper_math normalize on the host: v * (1 / sqrtf(dot(v, v))) in float */
    static float3 normalize_host(float3 v) {
        const float d = v.x * v.x + v.y * v.y + v.z * v.z;
        const float inv = 1.0f / std::sqrt(d);
        return float3{v.x * inv, v.y * inv, v.z * inv};
    }

    unsigned load_order;
    unsigned family_code = DEME_RESERVED_FAMILY;
    float3 init_pos{0.f, 0.f, 0.f};
    float mass = 1e15f;
    float3 MOI{1e15f, 1e15f, 1e15f};
    std::vector<DEMAnalEntity> entities;
};

/* DEMMeshConnected (src/DEM/BdrsAndObjs.h:173-300): a body represented by triangle facets given in its own frame.
 * Defaults as the reference's: the fixed family, mass 1, principal moments 1, at the origin, unit orientation.
 * Its sphere--mesh contacts (one per facet a sphere touches) are an addition: the reference detects none. */
class DEMMeshConnected {
  public:
    DEMMeshConnected() = default;
    explicit DEMMeshConnected(const std::string& file) {
        if (!LoadWavefrontMesh(file)) throw std::runtime_error("cannot read the mesh file " + file);
    }
    DEMMeshConnected(const std::string& file, const std::shared_ptr<DEMMaterial>& mat) : DEMMeshConnected(file) {
        SetMaterial(mat);
    }
    /* The records of a Wavefront OBJ file as the reference's parser reads them (OBJ::ParseLine,
     * src/core/utils/WavefrontMeshLoader.hpp:578-647, behind src/DEM/MeshUtils.cpp:44-112): `v` and `vn` records
     * with three coordinates (a float rounded from the decimal value), `f` records of three or more corners split
     * into fans about the first corner, with the corners' normal indices (`a//n`, `a/t/n`) kept three at a time;
     * tags in any letter case.  Where the reference misreads a record, this reads it as the OBJ format defines it:
     * a negative index counts back from the last record read (the reference subtracts one from it, leaving an index
     * outside the mesh), and a vertex or normal record with more numbers or a trailing '#' comment is kept with its
     * first three (the reference drops it, shifting every later index).  Texture coordinates are not kept.  False
     * when the file cannot be opened or a number cannot be read. */
    bool LoadWavefrontMesh(const std::string& file, bool load_normals = true, bool load_uv = false) {
        (void)load_uv;
        std::ifstream in(file);
        if (!in) return false;
        vertices.clear();
        normals.clear();
        face_v_indices.clear();
        face_n_indices.clear();
        std::vector<int> flat_n;
        std::string line;
        try {
            while (std::getline(in, line)) {
                const size_t hash = line.find('#');
                if (hash != std::string::npos) line.resize(hash);
                std::istringstream ls(line);
                std::string tag;
                if (!(ls >> tag)) continue;
                for (char& c : tag) c = (char)std::tolower((unsigned char)c);
                if (tag == "v" || tag == "vn") {
                    std::string x, y, z;
                    if (!(ls >> x >> y >> z)) continue;
                    const float3 p{(float)std::stod(x), (float)std::stod(y), (float)std::stod(z)};
                    (tag == "v" ? vertices : normals).push_back(p);
                } else if (tag == "f") {
                    std::vector<int> vi, ni;
                    std::string tok;
                    while (ls >> tok) {
                        const size_t s1 = tok.find('/');
                        const int i = std::stoi(tok.substr(0, s1));
                        vi.push_back(i > 0 ? i - 1 : (int)vertices.size() + i);
                        const size_t s2 = s1 == std::string::npos ? s1 : tok.find('/', s1 + 1);
                        if (s2 != std::string::npos && s2 + 1 < tok.size()) {
                            const int k = std::stoi(tok.substr(s2 + 1));
                            ni.push_back(k > 0 ? k - 1 : (int)normals.size() + k);
                        } else {
                            ni.push_back(INT_MIN);
                        }
                    }
                    for (size_t j = 1; j + 1 < vi.size(); j++) {
                        face_v_indices.push_back(int3{vi[0], vi[j], vi[j + 1]});
                        for (size_t c : {(size_t)0, j, j + 1})
                            if (ni[c] != INT_MIN) flat_n.push_back(ni[c]);
                    }
                }
            }
        } catch (const std::logic_error&) {
            return false;
        }
        for (size_t k = 0; k + 2 < flat_n.size(); k += 3) face_n_indices.push_back(int3{flat_n[k], flat_n[k + 1], flat_n[k + 2]});
        if (!load_normals) {
            normals.clear();
            face_n_indices.clear();
        }
        nTri = face_v_indices.size();
        return true;
    }
    size_t GetNumTriangles() const { return nTri; }
    /* the i-th facet's nodes (DEMTriangle p1, p2, p3 in the reference) */
    std::vector<float3> GetTriangle(size_t i) const {
        const int3 f = face_v_indices.at(i);
        return {vertices.at((size_t)f.x), vertices.at((size_t)f.y), vertices.at((size_t)f.z)};
    }
    void Clear() {
        vertices.clear();
        normals.clear();
        face_v_indices.clear();
        face_n_indices.clear();
        materials.clear();
        nTri = 0;
        isMaterialSet = false;
    }
    /* At initialisation, order each facet's nodes so that their right-hand normal agrees with the file's normal
     * at its first corner (src/DEM/APIPrivate.cpp:545-560; FacetNodes) */
    void UseNormals(bool use = true) { use_mesh_normals = use; }
    /* The i-th facet's nodes as initialisation places them: with UseNormals, nodes 2 and 3 swapped where
     * cross(p2 - p1, p3 - p1) points away from the normal of the first corner (float arithmetic, the reference's
     * float3 operators) */
    std::array<float3, 3> FacetNodes(size_t i) const {
        const int3 fv = face_v_indices.at(i);
        std::array<float3, 3> t{vertices.at((size_t)fv.x), vertices.at((size_t)fv.y), vertices.at((size_t)fv.z)};
        if (use_mesh_normals) {
            if (i >= face_n_indices.size())
                throw std::runtime_error("UseNormals needs a normal index for every facet of the mesh");
            const float3 n = normals.at((size_t)face_n_indices[i].x);
            const float3 ab{t[1].x - t[0].x, t[1].y - t[0].y, t[1].z - t[0].z};
            const float3 ac{t[2].x - t[0].x, t[2].y - t[0].y, t[2].z - t[0].z};
            const float cx = ab.y * ac.z - ab.z * ac.y, cy = ab.z * ac.x - ab.x * ac.z, cz = ab.x * ac.y - ab.y * ac.x;
            const float d = cx * n.x + cy * n.y;
            if (d + cz * n.z < 0.f) std::swap(t[1], t[2]);
        }
        return t;
    }
    void SetFamily(unsigned code) {
        if (code > 255) throw std::runtime_error("family number is larger than the max allowance 255");
        family_code = code;
    }
    void SetMass(float m) { mass = m; }
    void SetMOI(float3 moi) { MOI = moi; }
    void SetMaterial(const std::vector<std::shared_ptr<DEMMaterial>>& input) {
        if (input.size() != nTri)
            throw std::runtime_error("SetMaterial input argument must have length " + std::to_string(nTri) + " (not " +
                                     std::to_string(input.size()) + "), same as the number of triangle facets in the mesh.");
        materials = input;
        isMaterialSet = true;
    }
    void SetMaterial(const std::shared_ptr<DEMMaterial>& input) {
        SetMaterial(std::vector<std::shared_ptr<DEMMaterial>>(nTri, input));
    }
    void SetInitPos(float3 p) { init_pos = p; }
    void SetInitQuat(float4 q) { init_oriQ = q; }  // (x, y, z, w)
    void SetInitVel(float3 v) { init_vel = v; }
    void SetInitAngVel(float3 w) { init_angvel = w; }
    /* moves the nodes in the mesh's own frame */
    void Translate(float3 d) {
        for (auto& v : vertices) v = float3{v.x + d.x, v.y + d.y, v.z + d.z};
    }
    void Scale(float s) { Scale(float3{s, s, s}); }
    /* one factor per axis; the normals keep their direction on the scaled surface */
    void Scale(float3 s) {
        for (auto& v : vertices) v = float3{v.x * s.x, v.y * s.y, v.z * s.z};
        for (auto& n : normals) {
            const double x = (double)n.x / s.x, y = (double)n.y / s.y, z = (double)n.z / s.z;
            const double l = std::sqrt(x * x + y * y + z * z);
            n = float3{(float)(x / l), (float)(y / l), (float)(z / l)};
        }
    }
    /* rotates the nodes in the mesh's own frame by the unit quaternion q = (x, y, z, w) */
    void Rotate(float4 q) {
        const double w = q.w, x = q.x, y = q.y, z = q.z;
        const double R[3][3] = {{1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)},
                                {2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)},
                                {2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)}};
        for (std::vector<float3>* a : {&vertices, &normals})
            for (auto& v : *a) {
                const double p[3] = {v.x, v.y, v.z};
                v = float3{(float)(R[0][0] * p[0] + R[0][1] * p[1] + R[0][2] * p[2]),
                           (float)(R[1][0] * p[0] + R[1][1] * p[1] + R[1][2] * p[2]),
                           (float)(R[2][0] * p[0] + R[2][1] * p[1] + R[2][2] * p[2])};
            }
    }
    /* Volume (the mass at unit density), centroid and the moments of inertia about the centroid along the mesh's
     * axes, of the solid a closed, outward-wound mesh bounds (declared, not defined, in the reference:
     * BdrsAndObjs.h:291): the divergence theorem over each facet (Eberly's polyhedral mass properties), in double. */
    void ComputeMassProperties(double& mass, float3& center, float3& inertia) const {
        double m = 0, sx = 0, sy = 0, sz = 0, xx = 0, yy = 0, zz = 0;
        auto sub = [](double w0, double w1, double w2, double& f1, double& f2, double& f3) {
            const double t0 = w0 + w1;
            f1 = t0 + w2;
            const double t1 = w0 * w0;
            const double t2 = t1 + w1 * t0;
            f2 = t2 + w2 * f1;
            f3 = w0 * t1 + w1 * t2 + w2 * f2;
        };
        for (const int3& f : face_v_indices) {
            const float3 a = vertices.at((size_t)f.x), b = vertices.at((size_t)f.y), c = vertices.at((size_t)f.z);
            const double u[3] = {(double)b.x - a.x, (double)b.y - a.y, (double)b.z - a.z};
            const double v[3] = {(double)c.x - a.x, (double)c.y - a.y, (double)c.z - a.z};
            const double d[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
            double f1x, f2x, f3x, f1y, f2y, f3y, f1z, f2z, f3z;
            sub(a.x, b.x, c.x, f1x, f2x, f3x);
            sub(a.y, b.y, c.y, f1y, f2y, f3y);
            sub(a.z, b.z, c.z, f1z, f2z, f3z);
            m += d[0] * f1x;
            sx += d[0] * f2x;
            sy += d[1] * f2y;
            sz += d[2] * f2z;
            xx += d[0] * f3x;
            yy += d[1] * f3y;
            zz += d[2] * f3z;
        }
        m /= 6.0;
        const double cx = sx / 24.0 / m, cy = sy / 24.0 / m, cz = sz / 24.0 / m;
        xx /= 60.0;
        yy /= 60.0;
        zz /= 60.0;
        mass = m;
        center = float3{(float)cx, (float)cy, (float)cz};
        inertia = float3{(float)(yy + zz - m * (cy * cy + cz * cz)), (float)(zz + xx - m * (cz * cz + cx * cx)),
                         (float)(xx + yy - m * (cx * cx + cy * cy))};
    }
    /* WriteWavefront (src/DEM/MeshUtils.cpp:119-165): every mesh's vertices, then the normals of the meshes that have
     * them, then the faces offset into one object (`f a//n b//n c//n` for a mesh with normals) */
    static void WriteWavefront(const std::string& filename, std::vector<DEMMeshConnected>& meshes) {
        std::ofstream mf(filename);
        for (const auto& m : meshes)
            for (const auto& v : m.vertices) mf << "v " << v.x << " " << v.y << " " << v.z << "\n";
        for (const auto& m : meshes)
            for (const auto& v : m.normals) mf << "vn " << v.x << " " << v.y << " " << v.z << "\n";
        int off = 1, noff = 1;
        for (const auto& m : meshes) {
            if (!m.normals.empty()) {
                if (m.face_n_indices.size() != m.face_v_indices.size())
                    throw std::runtime_error("a mesh with normals needs one normal triple per facet");
                for (size_t j = 0; j < m.face_v_indices.size(); j++) {
                    const int3 f = m.face_v_indices[j], n = m.face_n_indices[j];
                    mf << "f " << f.x + off << "//" << n.x + noff << " " << f.y + off << "//" << n.y + noff << " "
                       << f.z + off << "//" << n.z + noff << "\n";
                }
            } else {
                for (const auto& f : m.face_v_indices)
                    mf << "f " << f.x + off << " " << f.y + off << " " << f.z + off << "\n";
            }
            off += (int)m.vertices.size();
            noff += (int)m.normals.size();
        }
    }
    /* One mesh of the given meshes' nodes, normals and facets (declared, not defined, in the reference:
     * BdrsAndObjs.h:250); the first mesh's body properties, no materials */
    static DEMMeshConnected Merge(std::vector<DEMMeshConnected>& meshes) {
        DEMMeshConnected out;
        if (!meshes.empty()) {
            out.mass = meshes[0].mass;
            out.MOI = meshes[0].MOI;
            out.family_code = meshes[0].family_code;
        }
        for (const auto& m : meshes) {
            const int vo = (int)out.vertices.size(), no = (int)out.normals.size();
            out.vertices.insert(out.vertices.end(), m.vertices.begin(), m.vertices.end());
            out.normals.insert(out.normals.end(), m.normals.begin(), m.normals.end());
            for (const int3& f : m.face_v_indices) out.face_v_indices.push_back(int3{f.x + vo, f.y + vo, f.z + vo});
            for (const int3& f : m.face_n_indices) out.face_n_indices.push_back(int3{f.x + no, f.y + no, f.z + no});
        }
        out.nTri = out.face_v_indices.size();
        return out;
    }

    size_t nTri = 0;
    std::vector<float3> vertices;
    std::vector<int3> face_v_indices;
    std::vector<float3> normals;
    std::vector<int3> face_n_indices;
    bool use_mesh_normals = false;
    std::vector<std::shared_ptr<DEMMaterial>> materials;
    bool isMaterialSet = false;
    unsigned family_code = DEME_RESERVED_FAMILY;
    float mass = 1.f;
    float3 MOI{1.f, 1.f, 1.f};
    float3 init_pos{0.f, 0.f, 0.f};
    float4 init_oriQ{0.f, 0.f, 0.f, 1.f};
    float3 init_vel{0.f, 0.f, 0.f};
    float3 init_angvel{0.f, 0.f, 0.f};
    unsigned load_order = 0;
};

class DEMForceModel {
  public:
    void DefineCustomModel(const std::string& model) { m_force_model = model; custom = true; }
    int ReadCustomModelFile(const std::string& path) {
        std::ifstream f(path);
        if (!f) return 1;
        std::stringstream ss;
        ss << f.rdbuf();
        DefineCustomModel(ss.str());
        return 0;
    }
    void SetPerContactWildcards(const std::set<std::string>& names) { m_contact_wildcards = names; }
    /* DEMForceModel::SetForceModelType (AuxClasses.cpp:218-236): the built-in full or frictionless Hertzian model
     * with its wildcards, or a custom one (its string comes from DefineCustomModel) */
    void SetForceModelType(FORCE_MODEL t) {
        custom = t == FORCE_MODEL::CUSTOM;
        frictionless = t == FORCE_MODEL::HERTZIAN_FRICTIONLESS;
        if (t == FORCE_MODEL::HERTZIAN)
            m_contact_wildcards = {"delta_tan_x", "delta_tan_y", "delta_tan_z", "delta_time"};
        else if (frictionless)
            m_contact_wildcards.clear();
    }

    bool custom = false;
    bool frictionless = false;  // UseFrictionlessHertzianModel: normal force only, no contact wildcards
    std::string m_force_model;
    std::set<std::string> m_contact_wildcards{"delta_tan_x", "delta_tan_y", "delta_tan_z", "delta_time"};
};

/* The flattened scene Initialize hands to deme_create (owned arrays; `scene` points into them). */
struct FlatScene {
    deme_sim_params params{};
    deme_scene scene{};
    std::vector<uint64_t> voxel;
    std::vector<uint16_t> locX, locY, locZ;
    std::vector<float> oriQw, oriQx, oriQy, oriQz, vX, vY, vZ, omgX, omgY, omgZ, mass, mmiXX, mmiYY, mmiZZ;
    std::vector<uint8_t> family;
    std::vector<uint32_t> sphere_owner;
    std::vector<float> relX, relY, relZ, radius;
    std::vector<uint8_t> sphere_material;
    std::vector<uint8_t> anal_type, anal_normal, anal_material;
    std::vector<uint32_t> anal_owner;
    std::vector<float> anal_relX, anal_relY, anal_relZ, anal_rotX, anal_rotY, anal_rotZ, anal_size1, anal_size2,
        anal_size3, anal_mass;
    std::vector<float> mat_E, mat_nu, mat_CoR, mat_mu, mat_Crr;
    std::vector<uint8_t> family_masks;
    std::vector<deme_family_prescription> prescriptions;
    std::vector<uint32_t> tri_owner;
    std::vector<float> tri_node1, tri_node2, tri_node3;
    std::vector<uint16_t> tri_material;
    // families whose prescription holds an expression: strings kept here, pointed to by `motion`
    std::vector<std::vector<std::string>> motion_strings;  // per entry: vX vY vZ wX wY wZ X Y Z ("none" = free)
    std::vector<deme_motion_expressions> motion;
    // clump owners' template marks and the templates' names (the clump file's clump_type column)
    std::vector<uint32_t> owner_template;
    std::vector<std::string> template_names;

    void point() {
        deme_scene& s = scene;
        s.n_owners = (uint32_t)voxel.size();
        s.n_spheres = (uint32_t)radius.size();
        s.n_anal = (uint32_t)anal_type.size();
        s.n_materials = (uint32_t)mat_E.size();
        s.voxel = voxel.data();
        s.locX = locX.data();
        s.locY = locY.data();
        s.locZ = locZ.data();
        s.oriQw = oriQw.data();
        s.oriQx = oriQx.data();
        s.oriQy = oriQy.data();
        s.oriQz = oriQz.data();
        s.vX = vX.data();
        s.vY = vY.data();
        s.vZ = vZ.data();
        s.omgX = omgX.data();
        s.omgY = omgY.data();
        s.omgZ = omgZ.data();
        s.family = family.data();
        s.mass = mass.data();
        s.mmiXX = mmiXX.data();
        s.mmiYY = mmiYY.data();
        s.mmiZZ = mmiZZ.data();
        s.sphere_owner = sphere_owner.data();
        s.relX = relX.data();
        s.relY = relY.data();
        s.relZ = relZ.data();
        s.radius = radius.data();
        s.sphere_material = sphere_material.data();
        s.anal_type = anal_type.data();
        s.anal_owner = anal_owner.data();
        s.anal_normal = anal_normal.data();
        s.anal_material = anal_material.data();
        s.anal_relX = anal_relX.data();
        s.anal_relY = anal_relY.data();
        s.anal_relZ = anal_relZ.data();
        s.anal_rotX = anal_rotX.data();
        s.anal_rotY = anal_rotY.data();
        s.anal_rotZ = anal_rotZ.data();
        s.anal_size1 = anal_size1.data();
        s.anal_size2 = anal_size2.data();
        s.anal_size3 = anal_size3.data();
        s.anal_mass = anal_mass.data();
        s.mat_E = mat_E.data();
        s.mat_nu = mat_nu.data();
        s.mat_CoR = mat_CoR.data();
        s.mat_mu = mat_mu.data();
        s.mat_Crr = mat_Crr.data();
        s.family_masks = family_masks.data();
        s.prescriptions = prescriptions.data();
        s.n_tris = (uint32_t)tri_owner.size();
        s.tri_owner = s.n_tris ? tri_owner.data() : nullptr;
        s.tri_node1 = s.n_tris ? tri_node1.data() : nullptr;
        s.tri_node2 = s.n_tris ? tri_node2.data() : nullptr;
        s.tri_node3 = s.n_tris ? tri_node3.data() : nullptr;
        s.tri_material = s.n_tris ? tri_material.data() : nullptr;
    }
};

// ---- CSV output in DEM-Engine's formats (writeSpheresAsCsv / writeClumpsAsCsv / writeContactsAsCsv,
// src/DEM/dT.cpp:896-1180).  Values are formed in float as the reference's host code forms them and printed as a
// default std::ostream prints a float.  Contact points are rotated with owner A's quaternion (the reference uses
// the quaternion of the owner whose index equals the contact's index).
// OUTPUT_CONTENT / CNT_OUTPUT_CONTENT bits (src/DEM/Defines.h:118-143)
namespace OUTPUT_CONTENT {
constexpr unsigned XYZ = 0, QUAT = 1, ABSV = 2, VEL = 4, ANG_VEL = 8, ACC = 16, ANG_ACC = 32, FAMILY = 64, MAT = 128;
}
namespace CNT_OUTPUT_CONTENT {
constexpr unsigned OWNERS = 0, FORCE = 1, POINT = 2, COMPONENT = 4, NORMAL = 8, TORQUE_ONLY_FORCE = 16;
}

// Owner state as deme_download_state fills it.
struct OwnerState {
    std::vector<uint64_t> voxel;
    std::vector<uint16_t> locX, locY, locZ;
    std::vector<float> oriQw, oriQx, oriQy, oriQz, vX, vY, vZ;
    std::vector<float> omgX, omgY, omgZ;  // angular velocity in the owner's frame
    std::vector<uint8_t> family;
    void resize(size_t n) {
        voxel.resize(n);
        locX.resize(n);
        locY.resize(n);
        locZ.resize(n);
        for (auto* v : {&oriQw, &oriQx, &oriQy, &oriQz, &vX, &vY, &vZ, &omgX, &omgY, &omgZ}) v->resize(n);
        family.resize(n);
    }
};

namespace csv_detail {
// hostVoxelIDToPosition<float> plus the domain's lower corner (src/DEM/HostSideHelpers.hpp:308-324)
inline float3 owner_com(const FlatScene& f, const OwnerState& st, size_t o) {
    const deme_sim_params& p = f.params;
    const uint64_t v = st.voxel[o];
    const uint64_t mx = (1ull << p.nvXp2) - 1, my = (1ull << p.nvYp2) - 1;
    const float vs = (float)p.voxel_size, l = (float)p.l;
    const float X = (float)(v & mx) * vs + (float)st.locX[o] * l;
    const float Y = (float)((v >> p.nvXp2) & my) * vs + (float)st.locY[o] * l;
    const float Z = (float)(v >> (p.nvXp2 + p.nvYp2)) * vs + (float)st.locZ[o] * l;
    return float3{X + p.lbf[0], Y + p.lbf[1], Z + p.lbf[2]};
}
// hostApplyOriQToVector3<float, float> (src/DEM/HostSideHelpers.hpp:384-394)
inline float3 rotate(float3 r, float Qw, float Qx, float Qy, float Qz) {
    const float X = (2.f * (Qw * Qw + Qx * Qx) - 1.f) * r.x + (2.f * (Qx * Qy - Qw * Qz)) * r.y +
                    (2.f * (Qx * Qz + Qw * Qy)) * r.z;
    const float Y = (2.f * (Qx * Qy + Qw * Qz)) * r.x + (2.f * (Qw * Qw + Qy * Qy) - 1.f) * r.y +
                    (2.f * (Qy * Qz - Qw * Qx)) * r.z;
    const float Z = (2.f * (Qx * Qz - Qw * Qy)) * r.x + (2.f * (Qy * Qz + Qw * Qx)) * r.y +
                    (2.f * (Qw * Qw + Qz * Qz) - 1.f) * r.z;
    return float3{X, Y, Z};
}
inline float speed(float x, float y, float z) { return std::sqrt(x * x + y * y + z * z); }
}  // namespace csv_detail

/* The reference's inspectors (DEMInspector, src/DEM/AuxClasses.cpp:14-106; inspectSphereProperty,
 * src/kernel/DEMSphereQueryKernels.cu:9-50), on an owner state, over the whole domain:
 *   "clump_max_z" / "clump_min_z": the largest sphere top / smallest sphere bottom, Z +- r, with the sphere centre
 *   formed as the kernel forms it (owner position in double from the voxel code and the kernel literals, the
 *   relative position rotated in float, the lower corner added, rounded to float);
 *   "clump_max_absv": the largest speed of a sphere centre, |v + R (omega x relPos)| in float;
 *   "clump_volume": the sum of the clumps' template volumes (DEMClumpTemplate::SetVolume, 0 unless set). */
inline float inspect_quantity(const FlatScene& f, const OwnerState& st, const std::string& q,
                              const std::vector<float>& template_volume) {
    using namespace csv_detail;
    const deme_sim_params& p = f.params;
    if (q == "clump_volume") {
        float sum = 0.f;
        for (size_t o = 0; o < f.owner_template.size(); o++)
            sum += f.owner_template[o] < template_volume.size() ? template_volume[f.owner_template[o]] : 0.f;
        return sum;
    }
    const bool top = q == "clump_max_z", bottom = q == "clump_min_z", absv = q == "clump_max_absv";
    if (!top && !bottom && !absv) throw std::runtime_error(q + " is not a known query type.");
    float best = bottom ? 3.4e38f : -3.4e38f;
    for (size_t i = 0; i < f.radius.size(); i++) {
        const size_t o = f.sphere_owner[i];
        const float qw = st.oriQw[o], qx = st.oriQx[o], qy = st.oriQy[o], qz = st.oriQz[o];
        float v;
        if (absv) {
            const float rx = f.relX[i], ry = f.relY[i], rz = f.relZ[i];
            const float wx = st.omgX[o], wy = st.omgY[o], wz = st.omgZ[o];
            const float3 w = rotate(float3{wy * rz - wz * ry, wz * rx - wx * rz, wx * ry - wy * rx}, qw, qx, qy, qz);
            v = speed(w.x + st.vX[o], w.y + st.vY[o], w.z + st.vZ[o]);
        } else {
            const float3 d = rotate(float3{f.relX[i], f.relY[i], f.relZ[i]}, qw, qx, qy, qz);
            const double oz = (double)(st.voxel[o] >> (p.nvXp2 + p.nvYp2)) * p.voxel_size_kernel +
                              (double)st.locZ[o] * p.l_kernel;
            const float Z = (float)(oz + (double)d.z + (double)p.lbf[2]);
            v = top ? Z + f.radius[i] : Z - f.radius[i];
        }
        best = bottom ? std::min(best, v) : std::max(best, v);
    }
    return best;
}

inline void write_sphere_csv(std::ostream& os, const FlatScene& f, const OwnerState& st, unsigned content,
                             const std::set<unsigned>& no_output = {}) {
    using namespace csv_detail;
    os << "X,Y,Z,r";
    if (content & OUTPUT_CONTENT::ABSV) os << ",absv";
    if (content & OUTPUT_CONTENT::VEL) os << ",v_x,v_y,v_z";
    if (content & OUTPUT_CONTENT::FAMILY) os << ",family";
    os << "\n";
    for (size_t i = 0; i < f.radius.size(); i++) {
        const size_t o = f.sphere_owner[i];
        if (no_output.count(st.family[o])) continue;
        const float3 c = owner_com(f, st, o);
        const float3 d = rotate(float3{f.relX[i], f.relY[i], f.relZ[i]}, st.oriQw[o], st.oriQx[o], st.oriQy[o],
                                st.oriQz[o]);
        os << c.x + d.x << "," << c.y + d.y << "," << c.z + d.z << "," << f.radius[i];
        if (content & OUTPUT_CONTENT::ABSV) os << "," << speed(st.vX[o], st.vY[o], st.vZ[o]);
        if (content & OUTPUT_CONTENT::VEL) os << "," << st.vX[o] << "," << st.vY[o] << "," << st.vZ[o];
        if (content & OUTPUT_CONTENT::FAMILY) os << "," << +st.family[o];
        os << "\n";
    }
}

inline void write_clump_csv(std::ostream& os, const FlatScene& f, const OwnerState& st, unsigned content,
                            const std::set<unsigned>& no_output = {}) {
    using namespace csv_detail;
    os << "X,Y,Z,Qw,Qx,Qy,Qz,clump_type";
    if (content & OUTPUT_CONTENT::ABSV) os << ",absv";
    if (content & OUTPUT_CONTENT::VEL) os << ",v_x,v_y,v_z";
    if (content & OUTPUT_CONTENT::FAMILY) os << ",family";
    os << "\n";
    for (size_t o = 0; o < f.owner_template.size(); o++) {
        if (no_output.count(st.family[o])) continue;
        const float3 c = owner_com(f, st, o);
        os << c.x << "," << c.y << "," << c.z << "," << st.oriQw[o] << "," << st.oriQx[o] << "," << st.oriQy[o]
           << "," << st.oriQz[o] << "," << f.template_names.at(f.owner_template[o]);
        if (content & OUTPUT_CONTENT::ABSV) os << "," << speed(st.vX[o], st.vY[o], st.vZ[o]);
        if (content & OUTPUT_CONTENT::VEL) os << "," << st.vX[o] << "," << st.vY[o] << "," << st.vZ[o];
        if (content & OUTPUT_CONTENT::FAMILY) os << "," << +st.family[o];
        os << "\n";
    }
}

// Contacts as deme_download_contacts gives them; force, torque-only force and A's local contact point (n x 3 each)
// as deme_download_contact_forces gives them.
inline void write_contact_csv(std::ostream& os, const FlatScene& f, const OwnerState& st,
                              const std::vector<uint32_t>& idA, const std::vector<uint32_t>& idB,
                              const std::vector<uint8_t>& type, const std::vector<float>& force,
                              const std::vector<float>& tof, const std::vector<float>& cpA, unsigned content) {
    using namespace csv_detail;
    os << "A,B,contact_type";
    if (content & CNT_OUTPUT_CONTENT::FORCE) os << ",f_x,f_y,f_z";
    if (content & CNT_OUTPUT_CONTENT::POINT) os << ",X,Y,Z";
    if (content & CNT_OUTPUT_CONTENT::NORMAL) os << ",n_x,n_y,n_z";
    if (content & CNT_OUTPUT_CONTENT::TORQUE_ONLY_FORCE) os << ",tof_x,tof_y,tof_z";
    os << "\n";
    for (size_t i = 0; i < idA.size(); i++) {
        if (type[i] == DEME_NOT_A_CONTACT) continue;
        const uint32_t oA = f.sphere_owner[idA[i]];
        const uint32_t oB = type[i] == DEME_SPHERE_SPHERE_CONTACT ? f.sphere_owner[idB[i]] : f.anal_owner[idB[i]];
        os << oA << "," << oB << "," << (type[i] == DEME_SPHERE_SPHERE_CONTACT ? "SS" : (type[i] == 2 ? "SM" : "SA"));
        if (content & CNT_OUTPUT_CONTENT::FORCE)
            os << "," << force[3 * i] << "," << force[3 * i + 1] << "," << force[3 * i + 2];
        const float3 c = owner_com(f, st, oA);
        float3 p = rotate(float3{cpA[3 * i], cpA[3 * i + 1], cpA[3 * i + 2]}, st.oriQw[oA], st.oriQx[oA],
                          st.oriQy[oA], st.oriQz[oA]);
        p = float3{c.x + p.x, c.y + p.y, c.z + p.z};
        if (content & CNT_OUTPUT_CONTENT::POINT) os << "," << p.x << "," << p.y << "," << p.z;
        if (content & CNT_OUTPUT_CONTENT::NORMAL) {
            const float3 d = rotate(float3{f.relX[idA[i]], f.relY[idA[i]], f.relZ[idA[i]]}, st.oriQw[oA],
                                    st.oriQx[oA], st.oriQy[oA], st.oriQz[oA]);
            float nx = p.x - (c.x + d.x), ny = p.y - (c.y + d.y), nz = p.z - (c.z + d.z);
            const float inv = 1.f / std::sqrt(nx * nx + ny * ny + nz * nz);
            os << "," << nx * inv << "," << ny * inv << "," << nz * inv;
        }
        if (content & CNT_OUTPUT_CONTENT::TORQUE_ONLY_FORCE)
            os << "," << tof[3 * i] << "," << tof[3 * i + 1] << "," << tof[3 * i + 2];
        os << "\n";
    }
}

class DEMSolver;

/* DEMTracker (src/DEM/AuxClasses.h:76-121, AuxClasses.cpp:166-212): get and set one tracked owner (a clump batch's
 * first clump plus an offset, an external object or a mesh body) through the solver's per-owner calls.  Owner ids are
 * the reference's numbering, resolved when first used (after Initialize). */
class DEMTracker {
  public:
    DEMTracker(DEMSolver* sys, const void* obj, int kind) : sys(sys), obj(obj), kind(kind) {}
    float3 Pos(size_t offset = 0);
    float3 AngVelLocal(size_t offset = 0);
    float3 Vel(size_t offset = 0);
    float4 OriQ(size_t offset = 0);
    float3 ContactAcc(size_t offset = 0);
    float3 ContactAngAccLocal(size_t offset = 0);
    void SetPos(float3 pos, size_t offset = 0);
    void SetAngVel(float3 angVel, size_t offset = 0);
    void SetVel(float3 vel, size_t offset = 0);
    void SetOriQ(float4 oriQ, size_t offset = 0);
    /* an extra acceleration for the next step only: there is no such input on this build's step (a persistent one
     * is a family prescription) */
    void AddAcc(float3, size_t = 0) {
        throw std::runtime_error("AddAcc is not supported here; prescribe the family's motion instead");
    }
    void ChangeClumpSizes(const std::vector<uint32_t>& ids, const std::vector<float>& factors);
    uint32_t OwnerID();  // the tracked owner's id in the reference's numbering

  private:
    DEMSolver* sys;
    const void* obj;
    int kind;  // 0 clump batch, 1 external object, 2 mesh body
};

/* DEMInspector (src/DEM/AuxClasses.h:42-74): one of the reference's reductions over the running solver's state
 * (inspect_quantity), read back to the host. */
class DEMInspector {
  public:
    DEMInspector(DEMSolver* sys, const std::string& quantity) : sys(sys), quantity(quantity) {}
    float GetValue();

  private:
    DEMSolver* sys;
    std::string quantity;
};

class DEMSolver {
  public:
    DEMSolver() = default;
    ~DEMSolver() {
        if (h) deme_destroy(h);
    }
    DEMSolver(const DEMSolver&) = delete;
    DEMSolver& operator=(const DEMSolver&) = delete;

    // ---- world ----
    void InstructBoxDomainDimension(float x, float y, float z) { box = float3{x, y, z}; has_box = true; }
    /* the voxel bit split and length unit given directly (APIPublic.cpp:94-114); the domain is then the voxel world */
    void InstructBoxDomainNumVoxel(unsigned char x, unsigned char y, unsigned char z, float len_unit = 1e-10f) {
        if ((unsigned)x + y + z != 64u)
            throw std::runtime_error("Please give voxel numbers (as powers of 2) along each direction such that they "
                                     "add up to 64.");
        explicit_nv[0] = x;
        explicit_nv[1] = y;
        explicit_nv[2] = z;
        explicit_l = len_unit;
        has_explicit_nv = true;
    }
    bool GetInitStatus() const { return h != nullptr; }
    double GetTimeStepSize() const { return h_step; }
    float GetExpandFactor() const { return flat ? flat->params.beta : expand_factor; }
    // reference tuning and diagnostics switches with no counterpart here (the contact list is always sorted, kernels
    // are compiled ahead of time, output is CSV): accepted so that reference programs compile, no effect
    void SetVerbosity(VERBOSITY) {}
    /* CSV only (the writers below); the reference's binary and ChPF formats are not written */
    void SetOutputFormat(OUTPUT_FORMAT f) {
        if (f != OUTPUT_FORMAT::CSV) throw std::runtime_error("only the CSV output format is written");
    }
    void SetContactOutputFormat(OUTPUT_FORMAT f) { SetOutputFormat(f); }
    void SetSortContactPairs(bool) {}
    void SetJitifyClumpTemplates(bool = true) {}
    void SetJitifyMassProperties(bool = true) {}
    void SetOneBinPerThread(bool = true) {}
    void UseCompactForceKernel(bool = true) {}
    void EnsureKernelErrMsgLineNum(bool = true) {}
    void InstructNumOwners(size_t) {}
    void ReleaseFlattenedArrays() {}
    void ShowThreadCollaborationStats() {}
    void ClearThreadCollaborationStats() {}
    // Stubs in the reference itself, kept with its behaviour: SetFamilyPrescribedQuaternion checks the family and
    // stores nothing (APIPublic.cpp:275-280), and PurgeFamily is empty (:869).
    void SetFamilyPrescribedQuaternion(unsigned fam, const std::string&) {
        if (fam > 255) throw std::runtime_error("family number should not be larger than 255");
    }
    void PurgeFamily(unsigned) {}
    /* APIPublic.cpp:844-862: the listed clumps' spheres scaled by the factors (owner ids in the reference's numbering) */
    void ChangeClumpSizes(const std::vector<uint32_t>& ids, const std::vector<float>& factors) {
        if (!h) throw std::runtime_error("ChangeClumpSizes operates on the running solver: call it after Initialize");
        if (ids.size() != factors.size()) throw std::runtime_error("ChangeClumpSizes: one factor per clump");
        std::vector<uint32_t> o(ids.size());
        for (size_t i = 0; i < ids.size(); i++) o[i] = handle_owner(ids[i]);
        check(deme_change_clump_sizes(h, (uint32_t)o.size(), o.data(), factors.data()));
    }
    /* Per-kernel device times (deme_kernel_timing / deme_kernel_times) stand in for the reference's kT and dT phase
     * timers (kT.h:179-181, dT.h:253-255).  Timing brackets every launch with events and keeps whole steps off CUDA
     * graphs, so it is off until this build's EnableTimingStats turns it on. */
    void EnableTimingStats(bool on = true) {
        check(deme_kernel_timing(on ? 1 : 0));
        timing_on = on;
    }
    void ClearTimingStats() {
        if (timing_on) check(deme_kernel_timing(1));
    }
    void ShowTimingStats() {
        const char* names[64];
        double ms[64];
        int64_t cnt[64];
        int32_t n = 0;
        check(deme_kernel_times(64, names, ms, cnt, &n));
        double total = 0.0;
        for (int i = 0; i < n; i++) total += ms[i];
        std::printf("\n~~ KERNEL TIMING STATISTICS ~~\n");
        if (!timing_on || total <= 0.0) {
            std::printf("no kernel timed (EnableTimingStats turns per-kernel timing on)\n");
            return;
        }
        std::printf("total device time: %.9g seconds\n", total / 1e3);
        for (int i = 0; i < n; i++)
            if (cnt[i] > 0)
                std::printf("%s: %.9g seconds over %lld launches, %.6g%% of the total\n", names[i], ms[i] / 1e3,
                            (long long)cnt[i], ms[i] / total * 100.);
    }
    void SetCoordSysOrigin(const std::string& where) { origin = where; }
    void SetCoordSysOrigin(float3 lbf) { LBF = lbf; origin = "explicit"; }
    void InstructBoxDomainBoundingBC(const std::string& inst, const std::shared_ptr<DEMMaterial>& mat) {
        bounding_bc = inst;
        bounding_mat = mat;
    }
    void SetGravitationalAcceleration(float3 g) { G = g; }
    void SetInitTimeStep(double ts) { h_step = ts; }
    void UpdateStepSize(double ts) {
        h_step = ts;
        if (h) check(deme_set_time_step(h, (float)ts));
    }
    /* after Initialize (APIPublic.cpp:786-790, which transfers the solver and simulation parameters again): the time
     * step is applied; gravity, the contact margin and the integrator are fixed when the solver is created, so a
     * change of them since Initialize is refused rather than ignored */
    void UpdateSimParams() {
        if (!h) throw std::runtime_error("UpdateSimParams: call it only after Initialize");
        const deme_sim_params& p = flat->params;
        if (p.G[0] != G.x || p.G[1] != G.y || p.G[2] != G.z || p.integrator != integrator ||
            (expand_fixed && p.beta != expand_factor))
            throw std::runtime_error("UpdateSimParams: only the time step can change after Initialize here");
        check(deme_set_time_step(h, (float)h_step));
    }
    void SetInitBinSize(double b) { bin_size = b; }
    void SetCDUpdateFreq(int f) { update_freq = f; }
    void SetExpandFactor(float beta, bool fix = true) { expand_factor = beta; expand_fixed = fix; }
    void SetMaxVelocity(float v) { max_vel = v; }
    void SetExpandSafetyParam(float s) { safety = s; }
    void SetIntegrator(TIME_INTEGRATOR t) { integrator = (int)t; }

    // ---- materials, templates, clumps, objects ----
    std::shared_ptr<DEMMaterial> LoadMaterial(const std::unordered_map<std::string, float>& props) {
        materials.push_back(std::make_shared<DEMMaterial>(props, (unsigned)materials.size()));
        return materials.back();
    }
    std::shared_ptr<DEMClumpTemplate> LoadClumpType(float mass, float3 moi, const std::vector<float>& radii,
                                                    const std::vector<float3>& relPos,
                                                    const std::vector<std::shared_ptr<DEMMaterial>>& mats) {
        if (radii.size() != relPos.size() || radii.size() != mats.size())
            throw std::runtime_error("LoadClumpType: radii, positions and materials differ in length");
        auto t = std::make_shared<DEMClumpTemplate>();
        t->mass = mass;
        t->MOI = moi;
        t->radii = radii;
        t->relPos = relPos;
        t->materials = mats;
        t->mark = (unsigned)templates.size();
        char name[16];
        std::snprintf(name, sizeof(name), "%04d", (int)templates.size());
        t->AssignName(name);
        templates.push_back(t);
        return t;
    }
    /* the template built by the caller (API.h:173) */
    std::shared_ptr<DEMClumpTemplate> LoadClumpType(DEMClumpTemplate& clump) {
        return LoadClumpType(clump.mass, clump.MOI, clump.radii, clump.relPos, clump.materials);
    }
    /* components from a CSV file (API.h:175-184; DEMClumpTemplate::ReadComponentFromFile) */
    std::shared_ptr<DEMClumpTemplate> LoadClumpType(float mass, float3 moi, const std::string& filename,
                                                    const std::vector<std::shared_ptr<DEMMaterial>>& mats) {
        DEMClumpTemplate c;
        if (c.ReadComponentFromFile(filename)) throw std::runtime_error("cannot read clump file " + filename);
        return LoadClumpType(mass, moi, c.radii, c.relPos, mats);
    }
    std::shared_ptr<DEMClumpTemplate> LoadClumpType(float mass, float3 moi, const std::string& filename,
                                                    const std::shared_ptr<DEMMaterial>& mat) {
        DEMClumpTemplate c;
        if (c.ReadComponentFromFile(filename)) throw std::runtime_error("cannot read clump file " + filename);
        return LoadClumpType(mass, moi, c.radii, c.relPos,
                             std::vector<std::shared_ptr<DEMMaterial>>(c.radii.size(), mat));
    }
    std::shared_ptr<DEMClumpTemplate> LoadClumpType(float mass, float3 moi, const std::vector<float>& radii,
                                                    const std::vector<float3>& relPos,
                                                    const std::shared_ptr<DEMMaterial>& mat) {
        return LoadClumpType(mass, moi, radii, relPos, std::vector<std::shared_ptr<DEMMaterial>>(radii.size(), mat));
    }
    /* APIPublic.cpp:402-409: MOI 2/5 m r^2 */
    std::shared_ptr<DEMClumpTemplate> LoadSphereType(float mass, float radius,
                                                     const std::shared_ptr<DEMMaterial>& mat) {
        const float I = (float)(2.0 / 5.0 * mass * radius * radius);
        return LoadClumpType(mass, float3{I, I, I}, {radius}, {float3{0.f, 0.f, 0.f}}, mat);
    }
    std::shared_ptr<DEMClumpBatch> AddClumps(const std::vector<std::shared_ptr<DEMClumpTemplate>>& types,
                                             const std::vector<float3>& xyz) {
        auto b = std::make_shared<DEMClumpBatch>(xyz.size());
        b->SetTypes(types);
        b->SetPos(xyz);
        batches.push_back(b);
        return b;
    }
    std::shared_ptr<DEMClumpBatch> AddClumps(const std::shared_ptr<DEMClumpTemplate>& type,
                                             const std::vector<float3>& xyz) {
        return AddClumps(std::vector<std::shared_ptr<DEMClumpTemplate>>(xyz.size(), type), xyz);
    }
    /* CreateInspector (API.h:248-249): "clump_max_z", "clump_min_z", "clump_max_absv" or "clump_volume" over the
     * whole domain; a region (a compiled expression of X, Y, Z in the reference) is not supported */
    std::shared_ptr<DEMInspector> CreateInspector(const std::string& quantity = "clump_max_z") {
        if (quantity != "clump_max_z" && quantity != "clump_min_z" && quantity != "clump_max_absv" &&
            quantity != "clump_volume")
            throw std::runtime_error(quantity + " is not a known query type.");
        return std::make_shared<DEMInspector>(this, quantity);
    }
    std::shared_ptr<DEMInspector> CreateInspector(const std::string&, const std::string&) {
        throw std::runtime_error("inspectors of a region are not supported here; inspect the whole domain");
    }
    float InspectValue(const std::string& quantity) {
        if (!h) throw std::runtime_error("Inspector should only be used after the simulation system is initialized");
        const OwnerState st = pull_owner_state();
        std::vector<float> vols;
        for (const auto& t : templates) vols.push_back(t->volume);
        return inspect_quantity(*flat, st, quantity, vols);
    }
    std::shared_ptr<DEMTracker> Track(const std::shared_ptr<DEMClumpBatch>& obj) {
        return std::make_shared<DEMTracker>(this, obj.get(), 0);
    }
    std::shared_ptr<DEMTracker> Track(const std::shared_ptr<DEMExternObj>& obj) {
        return std::make_shared<DEMTracker>(this, obj.get(), 1);
    }
    std::shared_ptr<DEMTracker> Track(const std::shared_ptr<DEMMeshConnected>& obj) {
        return std::make_shared<DEMTracker>(this, obj.get(), 2);
    }
    /* the reference's owner id of a batch's first clump, an external object or a mesh body */
    uint32_t TrackedOwnerID(const void* obj, int kind) const {
        if (!h) throw std::runtime_error("a tracker is read or written only after Initialize");
        size_t id = 0;
        if (kind == 0) {
            for (const auto& b : system_batches) {
                if (b.get() == obj) return (uint32_t)(id < n_clumps_init ? id : id + n_ext_init + n_mesh_init);
                id += b->nClumps;
            }
        } else if (kind == 1) {
            for (size_t e = 0; e < ext.size(); e++)
                if (ext[e].get() == obj) return (uint32_t)(n_clumps_init + e);
        } else {
            for (size_t m = 0; m < meshes.size(); m++)
                if (meshes[m].get() == obj) return (uint32_t)(n_clumps_init + n_ext_init + m);
        }
        throw std::runtime_error("the tracked object is not part of the initialized system");
    }

    std::shared_ptr<DEMExternObj> AddExternalObject() {
        ext.push_back(std::make_shared<DEMExternObj>((unsigned)ext.size()));
        return ext.back();
    }
    std::shared_ptr<DEMExternObj> AddBCPlane(float3 pos, float3 normal, const std::shared_ptr<DEMMaterial>& mat) {
        auto o = AddExternalObject();
        o->AddPlane(pos, normal, mat);
        return o;
    }
    /* a mesh-represented body (AddWavefrontMeshObject, src/DEM/API.h:231-238) */
    std::shared_ptr<DEMMeshConnected> AddWavefrontMeshObject(const std::string& filename,
                                                             const std::shared_ptr<DEMMaterial>& mat,
                                                             bool load_normals = true, bool load_uv = false) {
        auto m = std::make_shared<DEMMeshConnected>();
        if (!m->LoadWavefrontMesh(filename, load_normals, load_uv))
            throw std::runtime_error("cannot read the mesh file " + filename);
        m->SetMaterial(mat);
        return AddWavefrontMeshObject(m);
    }
    std::shared_ptr<DEMMeshConnected> AddWavefrontMeshObject(const std::string& filename, bool load_normals = true,
                                                             bool load_uv = false) {
        auto m = std::make_shared<DEMMeshConnected>();
        if (!m->LoadWavefrontMesh(filename, load_normals, load_uv))
            throw std::runtime_error("cannot read the mesh file " + filename);
        return AddWavefrontMeshObject(m);
    }
    std::shared_ptr<DEMMeshConnected> AddWavefrontMeshObject(DEMMeshConnected& mesh) {
        return AddWavefrontMeshObject(std::make_shared<DEMMeshConnected>(mesh));
    }
    std::shared_ptr<DEMMeshConnected> AddWavefrontMeshObject(const std::shared_ptr<DEMMeshConnected>& mesh) {
        mesh->load_order = (unsigned)meshes.size();
        meshes.push_back(mesh);
        return mesh;
    }

    // ---- families ----
    /* before Initialize: part of the scene; after it: written into the running solver's mask table at once, as the
     * reference does (APIPublic.cpp:431-449), and kept for a later UpdateClumps */
    void DisableContactBetweenFamilies(unsigned a, unsigned b) {
        const unsigned lo = std::min(a, b), hi = std::max(a, b);
        if ((1u + hi) * hi / 2u + lo >= 255u * 256u / 2u)
            throw std::runtime_error("family mask entry out of range (the mask table holds 32640 entries)");
        no_contact.emplace_back(a, b);
        if (h) check(deme_set_family_contact(h, a, b, 1));
    }
    /* after Initialize only (APIPublic.cpp:451-468): families are in contact unless disabled */
    void EnableContactBetweenFamilies(unsigned a, unsigned b) {
        if (!h)
            throw std::runtime_error("There is no need to call EnableContactBetweenFamilies before system "
                                     "initialization. All families have contacts with each other by default.");
        const unsigned lo = std::min(a, b), hi = std::max(a, b);
        no_contact.erase(std::remove_if(no_contact.begin(), no_contact.end(),
                                        [&](const std::pair<unsigned, unsigned>& p) {
                                            return std::min(p.first, p.second) == lo &&
                                                   std::max(p.first, p.second) == hi;
                                        }),
                         no_contact.end());
        check(deme_set_family_contact(h, a, b, 0));
    }
    void SetFamilyFixed(unsigned fam) {
        Presc p(fam);
        p.linVel = {"0", "0", "0"};
        p.rotVel = {"0", "0", "0"};
        p.linVelP = p.rotVelP = p.linPosP = p.rotPosP = true;
        presc.push_back(p);
    }
    void SetFamilyPrescribedLinVel(unsigned fam, const std::string& vx, const std::string& vy, const std::string& vz,
                                   bool dictate = true) {
        Presc p(fam);
        p.linVel = {vx, vy, vz};
        p.linVelP = p.rotVelP = dictate;
        presc.push_back(p);
    }
    void SetFamilyPrescribedAngVel(unsigned fam, const std::string& wx, const std::string& wy, const std::string& wz,
                                   bool dictate = true) {
        Presc p(fam);
        p.rotVel = {wx, wy, wz};
        p.linVelP = p.rotVelP = dictate;
        presc.push_back(p);
    }
    void SetFamilyPrescribedPosition(unsigned fam, const std::string& x, const std::string& y, const std::string& z) {
        Presc p(fam);
        p.linPos = {x, y, z};
        p.linPosP = p.rotPosP = true;
        presc.push_back(p);
    }

    // ---- family changes (ChangeFamilyWhen / ChangeFamily, src/DEM/API.h:282-286) ----
    /* Rules are compiled at Initialize and applied every step after the forces. */
    void ChangeFamilyWhen(unsigned from, unsigned to, const std::string& condition) {
        fam_rules.push_back({from, to, condition});
    }
    void ChangeFamily(unsigned from, unsigned to) { check(deme_change_family(h, from, to)); }

    // ---- force model ----
    std::shared_ptr<DEMForceModel> UseFrictionalHertzianModel() {
        force_model = std::make_shared<DEMForceModel>();
        return force_model;
    }
    /* the frictionless Hertzian model (FrictionlessHertzianForceModel.cu): the built-in model with no contact
     * wildcards runs its normal part only */
    std::shared_ptr<DEMForceModel> UseFrictionlessHertzianModel() {
        force_model = std::make_shared<DEMForceModel>();
        force_model->frictionless = true;
        force_model->m_contact_wildcards.clear();
        return force_model;
    }
    std::shared_ptr<DEMForceModel> DefineContactForceModel(const std::string& model) {
        force_model = std::make_shared<DEMForceModel>();
        force_model->DefineCustomModel(model);
        force_model->m_contact_wildcards.clear();
        return force_model;
    }
    std::shared_ptr<DEMForceModel> ReadContactForceModel(const std::string& path) {
        force_model = std::make_shared<DEMForceModel>();
        force_model->m_contact_wildcards.clear();
        if (force_model->ReadCustomModelFile(path)) throw std::runtime_error("cannot read force model file " + path);
        return force_model;
    }

    // ---- lifecycle ----
    /* The scene as last flattened (by Flatten or Initialize). */
    const FlatScene& GetFlatScene() const { return *flat; }
    /* Flattens the scene (what Initialize uploads); usable without a GPU.  Initialize flattens again, which
     * replaces the FlatScene a previous call returned. */
    const FlatScene& Flatten() {
        flat = std::make_unique<FlatScene>();
        build_flat(*flat, batches);
        return *flat;
    }
    void Initialize() {
        system_batches = batches;
        create_handle();
        // after the flattening, which may add the bounding-box object
        n_clumps_init = n_clumps_system;
        n_ext_init = ext.size();
        n_mesh_init = meshes.size();
        n_templates_init = templates.size();
        n_materials_init = materials.size();
        n_presc_init = presc.size();
    }

    /* dT's cycle loop (src/DEM/dT.cpp:1527): steps while the accumulated time is below the duration */
    void DoDynamics(double duration) {
        const double hs = (double)flat->params.h;
        int32_t n = 0;
        for (double t = 0.0; t < duration; t += hs) n++;
        if (n) check(deme_step(h, n));
    }
    void DoDynamicsThenSync(double duration) {
        DoDynamics(duration);
        check(deme_sync(h));
    }
    void DoStepDynamics() { check(deme_step(h, 1)); }

  private:
    // Flattens the system (the batches in it, in order) and creates the handle with everything Initialize sets.
    void create_handle() {
        flat = std::make_unique<FlatScene>();
        build_flat(*flat, system_batches);
        n_clumps_system = 0;
        for (const auto& b : system_batches) n_clumps_system += b->nClumps;
        if (h) {
            deme_destroy(h);
            h = nullptr;
        }
        const int32_t st = deme_create(&flat->params, &flat->scene, &h);
        if (st != DEME_OK) {
            std::string msg = h ? deme_get_error(h) : "";
            if (h) deme_destroy(h);
            h = nullptr;
            throw std::runtime_error(std::string("Initialize: ") + deme_status_string(st) + ": " + msg);
        }
        if (cnt_out_content != CNT_OUTPUT_CONTENT::OWNERS) check(deme_keep_contact_forces(h, 1));
        if (!fam_rules.empty()) {
            std::vector<uint32_t> from, to;
            std::vector<const char*> cond;
            for (const auto& r : fam_rules) {
                from.push_back(r.from);
                to.push_back(r.to);
                cond.push_back(r.condition.c_str());
            }
            check(deme_set_family_change_rules(h, (int32_t)fam_rules.size(), from.data(), to.data(), cond.data()));
        }
        if (!flat->motion.empty()) {
            for (size_t i = 0; i < flat->motion.size(); i++) {
                const std::vector<std::string>& x = flat->motion_strings[i];
                deme_motion_expressions& me = flat->motion[i];
                auto str = [&](int j) { return x[j] == "none" ? nullptr : x[j].c_str(); };
                for (int k = 0; k < 3; k++) {
                    me.lin_vel[k] = str(k);
                    me.ang_vel[k] = str(3 + k);
                    me.lin_pos[k] = str(6 + k);
                }
            }
            check(deme_set_prescribed_motion(h, (int32_t)flat->motion.size(), flat->motion.data()));
        }
        if (force_model && force_model->custom) {
            std::vector<const char*> names;
            for (const auto& n : force_model->m_contact_wildcards) names.push_back(n.c_str());
            check(deme_set_force_model(h, force_model->m_force_model.c_str(), names.data(), (int32_t)names.size()));
        }
    }

  public:
    // ---- output (WriteSphereFile / WriteClumpFile / WriteContactFile, src/DEM/API.h:319-324, 430-436) ----
    void SetOutputContent(unsigned content) { out_content = content; }
    void SetContactOutputContent(unsigned content) { cnt_out_content = content; }
    void DisableFamilyOutput(unsigned fam) { no_output.insert(fam); }
    void WriteSphereFile(const std::string& path) {
        std::ofstream os(path);
        write_sphere_csv(os, *flat, pull_owner_state(), out_content, no_output);
    }
    void WriteClumpFile(const std::string& path) {
        std::ofstream os(path);
        write_clump_csv(os, *flat, pull_owner_state(), out_content, no_output);
    }
    /* Needs the per-contact forces of the last step: kept from Initialize on unless the contact output content was
     * set to owners only before it. */
    void WriteContactFile(const std::string& path) {
        uint32_t n = 0;
        check(deme_get_num_contacts(h, &n));
        const size_t cap = std::max<size_t>(n, 1);
        std::vector<uint32_t> idA(cap), idB(cap), map(cap);
        std::vector<uint8_t> type(cap);
        deme_contacts c{};
        c.capacity = (uint32_t)cap;
        c.idA = idA.data();
        c.idB = idB.data();
        c.type = type.data();
        c.mapping = map.data();
        check(deme_download_contacts(h, &c));
        idA.resize(n);
        idB.resize(n);
        type.resize(n);
        std::vector<float> F(3 * cap, 0.f), T(3 * cap, 0.f), P(3 * cap, 0.f);
        if (cnt_out_content != CNT_OUTPUT_CONTENT::OWNERS) {
            deme_contact_forces cf{};
            cf.capacity = (uint32_t)cap;
            cf.force = F.data();
            cf.torque_only_force = T.data();
            cf.cpA = P.data();
            check(deme_download_contact_forces(h, &cf));
        }
        std::ofstream os(path);
        write_contact_csv(os, *flat, pull_owner_state(), idA, idB, type, F, T, P, cnt_out_content);
    }

    /* ReadClumpXyzFromCsv / ReadClumpQuatFromCsv (src/DEM/API.h:326-371): clump type name -> coordinates or
     * quaternions (w, x, y, z) from a clump file, in file order, the numbers formed as the reference's reader
     * forms them (csv_float). */
    static std::unordered_map<std::string, std::vector<float3>> ReadClumpXyzFromCsv(
        const std::string& path, const std::string& clump_header = "clump_type", const std::string& x_header = "X",
        const std::string& y_header = "Y", const std::string& z_header = "Z") {
        std::unordered_map<std::string, std::vector<float3>> out;
        for (const auto& r : read_csv_columns(path, {clump_header, x_header, y_header, z_header}))
            out[r[0]].push_back(float3{csv_float(r[1]), csv_float(r[2]), csv_float(r[3])});
        return out;
    }
    static std::unordered_map<std::string, std::vector<float4>> ReadClumpQuatFromCsv(
        const std::string& path, const std::string& clump_header = "clump_type", const std::string& qw_header = "Qw",
        const std::string& qx_header = "Qx", const std::string& qy_header = "Qy", const std::string& qz_header = "Qz") {
        std::unordered_map<std::string, std::vector<float4>> out;
        for (const auto& r : read_csv_columns(path, {clump_header, qw_header, qx_header, qy_header, qz_header})) {
            float4 q;
            q.w = csv_float(r[1]);
            q.x = csv_float(r[2]);
            q.y = csv_float(r[3]);
            q.z = csv_float(r[4]);
            out[r[0]].push_back(q);
        }
        return out;
    }

    // ---- owner state (GetOwner* / SetOwner*, src/DEM/API.h:194-214; dT::getOwnerPos and its siblings,
    // src/DEM/dT.cpp:1705-1810).  Owner ids are the reference's: clumps of the first Initialize, then the external
    // objects, then the clumps each UpdateClumps added, in order. ----
    float3 GetOwnerPosition(uint32_t owner) {
        const One o = one(owner);
        const deme_sim_params& p = flat->params;
        const uint64_t mx = (1ull << p.nvXp2) - 1, my = (1ull << p.nvYp2) - 1;
        const double X = (double)(o.voxel & mx) * p.voxel_size + (double)o.loc[0] * p.l;
        const double Y = (double)((o.voxel >> p.nvXp2) & my) * p.voxel_size + (double)o.loc[1] * p.l;
        const double Z = (double)(o.voxel >> (p.nvXp2 + p.nvYp2)) * p.voxel_size + (double)o.loc[2] * p.l;
        return float3{(float)(X + p.lbf[0]), (float)(Y + p.lbf[1]), (float)(Z + p.lbf[2])};
    }
    float3 GetOwnerVelocity(uint32_t owner) {
        const One o = one(owner);
        return float3{o.f[0], o.f[1], o.f[2]};
    }
    float3 GetOwnerAngVel(uint32_t owner) {
        const One o = one(owner);
        return float3{o.f[3], o.f[4], o.f[5]};
    }
    float4 GetOwnerOriQ(uint32_t owner) {
        const One o = one(owner);
        return float4{o.f[7], o.f[8], o.f[9], o.f[6]};
    }
    /* Linear and angular acceleration from the contacts of the last step (gravity not included), as the
     * reference's aX / alphaX hold them after its force collection. */
    float3 GetOwnerAcc(uint32_t owner) {
        const One o = one(owner);
        return float3{o.f[10], o.f[11], o.f[12]};
    }
    float3 GetOwnerAngAcc(uint32_t owner) {
        const One o = one(owner);
        return float3{o.f[13], o.f[14], o.f[15]};
    }
    /* setOwnerPos: the position relative to the domain's lower corner, encoded on the voxel grid
     * (hostPositionToVoxelID, src/DEM/HostSideHelpers.hpp:328-350). */
    void SetOwnerPosition(uint32_t owner, float3 pos) {
        const deme_sim_params& p = flat->params;
        const double X = (double)(pos.x - p.lbf[0]), Y = (double)(pos.y - p.lbf[1]), Z = (double)(pos.z - p.lbf[2]);
        uint64_t voxel = 0;
        uint16_t loc[3];
        encode_position(p, X, Y, Z, voxel, loc);
        deme_state s{};
        s.voxel = &voxel;
        s.locX = &loc[0];
        s.locY = &loc[1];
        s.locZ = &loc[2];
        check(deme_upload_state_range(h, handle_owner(owner), 1, &s));
    }
    void SetOwnerVelocity(uint32_t owner, float3 vel) {
        deme_state s{};
        s.vX = &vel.x;
        s.vY = &vel.y;
        s.vZ = &vel.z;
        check(deme_upload_state_range(h, handle_owner(owner), 1, &s));
    }
    void SetOwnerAngVel(uint32_t owner, float3 angVel) {
        deme_state s{};
        s.omgX = &angVel.x;
        s.omgY = &angVel.y;
        s.omgZ = &angVel.z;
        check(deme_upload_state_range(h, handle_owner(owner), 1, &s));
    }
    void SetOwnerOriQ(uint32_t owner, float4 oriQ) {
        deme_state s{};
        s.oriQw = &oriQ.w;
        s.oriQx = &oriQ.x;
        s.oriQy = &oriQ.y;
        s.oriQz = &oriQ.z;
        check(deme_upload_state_range(h, handle_owner(owner), 1, &s));
    }

    // ---- adding clumps to a running simulation (ClearCache / UpdateClumps, src/DEM/APIPublic.cpp:470-490,
    // 792-843) ----
    /* Forgets the cached clump batches, so that a following AddClumps + UpdateClumps adds only the new ones.  The
     * clumps already in the simulation stay. */
    void ClearCache() { batches.clear(); }
    /* Adds every currently cached clump batch to the simulation: the clumps and spheres already there keep their
     * state, contact history and ids (new spheres follow the old ones), the simulation time carries on, and the
     * new clumps start from the state their batches give.  As in the reference, new clump templates, external
     * objects, materials or family prescriptions since Initialize are refused; without a ClearCache the clumps
     * cached before Initialize are added a second time. */
    void UpdateClumps() {
        if (!h) throw std::runtime_error("UpdateClumps: call it only after Initialize");
        if (ext.size() != n_ext_init || meshes.size() != n_mesh_init)
            throw std::runtime_error("UpdateClumps cannot be used after loading new analytical or mesh objects");
        if (templates.size() != n_templates_init)
            throw std::runtime_error("UpdateClumps cannot be used after loading new clump templates");
        if (materials.size() != n_materials_init || presc.size() != n_presc_init)
            throw std::runtime_error("UpdateClumps should not be used if you introduce new material types or family "
                                     "prescriptions");
        // the run so far: owner state, contact list with its history, time
        const uint32_t nO_old = flat->scene.n_owners;
        const size_t nC_old = n_clumps_system;
        OwnerState st = pull_owner_state();
        std::vector<float> omg[3];
        for (auto& v : omg) v.resize(nO_old);
        {
            deme_state s{};
            s.omgX = omg[0].data();
            s.omgY = omg[1].data();
            s.omgZ = omg[2].data();
            check(deme_download_state(h, &s));
        }
        uint32_t nc = 0;
        check(deme_get_num_contacts(h, &nc));
        const uint32_t cap = std::max<uint32_t>(nc, 1);
        const int nw = (force_model && force_model->custom) ? (int)force_model->m_contact_wildcards.size()
                                                             : flat->params.n_contact_wildcards;
        std::vector<uint32_t> idA(cap), idB(cap), map(cap);
        std::vector<uint8_t> type(cap);
        std::vector<float> wc((size_t)std::max(nw, 1) * cap);
        deme_contacts c{};
        c.capacity = cap;
        c.idA = idA.data();
        c.idB = idB.data();
        c.type = type.data();
        c.mapping = map.data();
        c.wildcards = nw ? wc.data() : nullptr;
        check(deme_download_contacts(h, &c));
        double t = 0.0;
        float tf = 0.f;
        int64_t steps = 0;
        check(deme_get_time(h, &t, &steps));
        check(deme_get_time_float(h, &tf));
        // the system grows by the cached batches; flatten and create the new handle as Initialize does
        for (const auto& b : batches) system_batches.push_back(b);
        create_handle();
        // carry the run over: old clumps keep their ids, the external and mesh objects move behind the new clumps
        const size_t nC_new = n_clumps_system, nExt = ext.size() + meshes.size();
        FlatScene& f = *flat;
        std::vector<uint64_t> voxel = f.voxel;
        std::vector<uint16_t> lx = f.locX, ly = f.locY, lz = f.locZ;
        std::vector<float> qw = f.oriQw, qx = f.oriQx, qy = f.oriQy, qz = f.oriQz, vx = f.vX, vy = f.vY, vz = f.vZ,
                           wx = f.omgX, wy = f.omgY, wz = f.omgZ;
        std::vector<uint8_t> fam = f.family;
        auto carry = [&](size_t from, size_t to) {
            voxel[to] = st.voxel[from];
            lx[to] = st.locX[from];
            ly[to] = st.locY[from];
            lz[to] = st.locZ[from];
            qw[to] = st.oriQw[from];
            qx[to] = st.oriQx[from];
            qy[to] = st.oriQy[from];
            qz[to] = st.oriQz[from];
            vx[to] = st.vX[from];
            vy[to] = st.vY[from];
            vz[to] = st.vZ[from];
            wx[to] = omg[0][from];
            wy[to] = omg[1][from];
            wz[to] = omg[2][from];
            fam[to] = st.family[from];
        };
        for (size_t o = 0; o < nC_old; o++) carry(o, o);
        for (size_t e = 0; e < nExt; e++) carry(nC_old + e, nC_new + e);
        deme_state s{};
        s.voxel = voxel.data();
        s.locX = lx.data();
        s.locY = ly.data();
        s.locZ = lz.data();
        s.oriQw = qw.data();
        s.oriQx = qx.data();
        s.oriQy = qy.data();
        s.oriQz = qz.data();
        s.vX = vx.data();
        s.vY = vy.data();
        s.vZ = vz.data();
        s.omgX = wx.data();
        s.omgY = wy.data();
        s.omgZ = wz.data();
        s.family = fam.data();
        check(deme_upload_state(h, &s));
        // sphere ids of the old clumps are unchanged (new spheres follow them), as are analytical component ids,
        // so the contact list and its history carry over as they are
        c.n_contacts = nc;
        if (nc) check(deme_upload_contacts(h, &c));
        check(deme_set_time(h, t, tf, steps));
    }

    uint32_t GetNumContacts() {
        uint32_t n = 0;
        check(deme_get_num_contacts(h, &n));
        return n;
    }
    double GetTotalKineticEnergy() {
        double ke = 0;
        check(deme_kinetic_energy(h, &ke));
        return ke;
    }
    /* the clumps' kinetic energy (API.h:315): the energy above already sums clump owners only */
    double GetClumpKineticEnergy() { return GetTotalKineticEnergy(); }
    double GetSimTime() {
        double t = 0;
        int64_t s = 0;
        check(deme_get_time(h, &t, &s));
        return t;
    }
    deme_handle* GetHandle() const { return h; }

  private:
    struct Presc {
        explicit Presc(unsigned f) : family(f) {}
        unsigned family;
        std::vector<std::string> linPos{"none", "none", "none"}, linVel{"none", "none", "none"},
            rotVel{"none", "none", "none"};
        bool linVelP = false, rotVelP = false, linPosP = false, rotPosP = false;
    };

    void check(int32_t st) {
        if (st != DEME_OK) throw std::runtime_error(std::string(deme_status_string(st)) + ": " + deme_get_error(h));
    }

    OwnerState pull_owner_state() {
        OwnerState st;
        const uint32_t n = flat->scene.n_owners;
        st.resize(n);
        deme_state s{};
        s.voxel = st.voxel.data();
        s.locX = st.locX.data();
        s.locY = st.locY.data();
        s.locZ = st.locZ.data();
        s.oriQw = st.oriQw.data();
        s.oriQx = st.oriQx.data();
        s.oriQy = st.oriQy.data();
        s.oriQz = st.oriQz.data();
        s.vX = st.vX.data();
        s.vY = st.vY.data();
        s.vZ = st.vZ.data();
        s.omgX = st.omgX.data();
        s.omgY = st.omgY.data();
        s.omgZ = st.omgZ.data();
        s.family = st.family.data();
        check(deme_download_state(h, &s));
        return st;
    }
    static std::vector<std::vector<std::string>> read_csv_columns(const std::string& path,
                                                                  const std::vector<std::string>& headers) {
        std::ifstream in(path);
        if (!in) throw std::runtime_error("cannot open " + path);
        auto split = [](const std::string& line) {
            std::vector<std::string> cells;
            std::stringstream ss(line);
            std::string c;
            while (std::getline(ss, c, ',')) {
                const size_t a = c.find_first_not_of(" \t\r"), b = c.find_last_not_of(" \t\r");
                cells.push_back(a == std::string::npos ? std::string() : c.substr(a, b - a + 1));
            }
            return cells;
        };
        std::string line;
        std::vector<std::string> head;
        while (head.empty() && std::getline(in, line))
            if (line.find_first_not_of(" \t\r") != std::string::npos) head = split(line);
        std::vector<size_t> idx;
        for (const auto& hname : headers) {
            const auto it = std::find(head.begin(), head.end(), hname);
            if (it == head.end()) throw std::runtime_error("column " + hname + " missing from " + path);
            idx.push_back((size_t)(it - head.begin()));
        }
        std::vector<std::vector<std::string>> rows;
        while (std::getline(in, line)) {
            if (line.find_first_not_of(" \t\r") == std::string::npos) continue;
            const auto cells = split(line);
            std::vector<std::string> r;
            for (size_t k : idx) r.push_back(k < cells.size() ? cells[k] : std::string());
            rows.push_back(r);
        }
        return rows;
    }

    // hostPositionToVoxelID (src/DEM/HostSideHelpers.hpp:328-350) for a position relative to the lower corner;
    // positions outside the voxel world clamp to its faces instead of wrapping.
    static void encode_position(const uint8_t nv[3], double voxel_size, double l, double X, double Y, double Z,
                                uint64_t& voxel, uint16_t sub[3]) {
        const double p[3] = {X, Y, Z};
        uint64_t n[3];
        for (int a = 0; a < 3; a++) {
            double q = p[a] / voxel_size;
            if (!(q > 0)) q = 0.0;
            n[a] = (uint64_t)std::floor(q);
            double u = (p[a] - (double)n[a] * voxel_size) / l;
            if (!(u > 0)) u = 0.0;
            u = std::min(u, 65535.0);
            sub[a] = (uint16_t)std::floor(u);
        }
        voxel = n[0] + (n[1] << nv[0]) + (n[2] << (nv[0] + nv[1]));
    }
    static void encode_position(const deme_sim_params& p, double X, double Y, double Z, uint64_t& voxel,
                                uint16_t sub[3]) {
        const uint8_t nv[3] = {p.nvXp2, p.nvYp2, p.nvZp2};
        encode_position(nv, p.voxel_size, p.l, X, Y, Z, voxel, sub);
    }

    // The handle's index of a reference owner id: the reference numbers the clumps of the first Initialize, then
    // the external objects and the mesh objects, then the clumps of each UpdateClumps; the handle keeps every clump
    // before the external and mesh objects.
    uint32_t handle_owner(uint32_t owner) const {
        const size_t nExt = n_ext_init + n_mesh_init;
        const uint32_t nO = flat ? flat->scene.n_owners : 0;
        uint32_t o = owner;
        if (owner >= n_clumps_init && owner < n_clumps_init + nExt)
            o = (uint32_t)(n_clumps_system + (owner - n_clumps_init));
        else if (owner >= n_clumps_init + nExt)
            o = (uint32_t)(owner - nExt);
        if (!h || o >= nO) throw std::runtime_error("owner id " + std::to_string(owner) + " out of range");
        return o;
    }

    // One owner's state (a ranged download of one entry).
    struct One {
        uint64_t voxel = 0;
        uint16_t loc[3] = {0, 0, 0};
        float f[16] = {};  // v, omega, q (w, x, y, z), a, alpha
    };
    One one(uint32_t owner) {
        One o;
        deme_state s{};
        s.voxel = &o.voxel;
        s.locX = &o.loc[0];
        s.locY = &o.loc[1];
        s.locZ = &o.loc[2];
        float* f = o.f;
        s.vX = f + 0;
        s.vY = f + 1;
        s.vZ = f + 2;
        s.omgX = f + 3;
        s.omgY = f + 4;
        s.omgZ = f + 5;
        s.oriQw = f + 6;
        s.oriQx = f + 7;
        s.oriQy = f + 8;
        s.oriQz = f + 9;
        s.aX = f + 10;
        s.aY = f + 11;
        s.aZ = f + 12;
        s.alphaX = f + 13;
        s.alphaY = f + 14;
        s.alphaZ = f + 15;
        check(deme_download_state_range(h, handle_owner(owner), 1, &s));
        return o;
    }

    static double kernel_literal(double x) {  // std::fixed, 17 decimals, parsed back (APIPrivate.cpp:1358-1359)
        char buf[128];
        std::snprintf(buf, sizeof(buf), "%.17f", x);
        return std::strtod(buf, nullptr);
    }
    /* a prescription string that is a plain number; anything else is an expression compiled at Initialize */
    static bool constant_expr(const std::string& e, double& v) {
        char* end = nullptr;
        v = std::strtod(e.c_str(), &end);
        while (end && *end == ' ') end++;
        return end && end != e.c_str() && *end == '\0';
    }

    /* figureOutNV, src/DEM/APIPrivate.cpp:222-333 (no exact direction) */
    void figure_out_nv(uint8_t nv[3], double& l) const {
        float XYZ[3] = {box.x, box.y, box.z};
        int rank[3] = {0, 1, 2};
        for (int i = 0; i < 2; i++)
            for (int j = i + 1; j < 3; j++)
                if (XYZ[i] > XYZ[j]) {
                    std::swap(XYZ[i], XYZ[j]);
                    std::swap(rank[i], rank[j]);
                }
        const float size321[3] = {XYZ[0], XYZ[1], XYZ[2]};
        int more[2] = {0, 0};
        for (int a = 0; a < 2; a++) {
            while (XYZ[a] < XYZ[a + 1]) {
                if (std::sqrt(2.0) * (double)XYZ[a] > (double)XYZ[a + 1]) break;
                more[a]++;
                XYZ[a] = (float)((double)XYZ[a] * 2.0);
            }
        }
        const int base = (64 - more[0] - more[1]) / 3;
        int left = (64 - more[0] - more[1]) % 3;
        int b3 = base, b2 = b3 + more[0], b1 = b2 + more[1];
        while (left > 0) {
            if (b3 < b2)
                b3++;
            else if (b2 < b1)
                b2++;
            else
                b1++;
            left--;
        }
        const int bits[3] = {b3, b2, b1};
        if (b1 + b2 + b3 > 64)
            throw std::runtime_error("domain needs more than 64 voxel bits under the reference's bit split; use a "
                                     "domain whose two smaller sides are within a factor sqrt(2)");
        double lmax = 0.0;
        for (int i = 0; i < 3; i++) lmax = std::max(lmax, (double)size321[i] / 65536.0 / std::ldexp(1.0, bits[i]));
        l = (double)(float)lmax;
        for (int i = 0; i < 3; i++) nv[rank[i]] = (uint8_t)bits[i];
    }

    void build_flat(FlatScene& f, const std::vector<std::shared_ptr<DEMClumpBatch>>& batches) {
        if (!has_box && !has_explicit_nv)
            throw std::runtime_error("InstructBoxDomainDimension must be called before Initialize");
        uint8_t nv[3];
        double l = 0.0;
        if (has_explicit_nv) {
            for (int a = 0; a < 3; a++) nv[a] = explicit_nv[a];
            l = (double)explicit_l;
            const double vox = 65536.0 * l;
            box = float3{(float)(vox * (double)(1ull << nv[0])), (float)(vox * (double)(1ull << nv[1])),
                         (float)(vox * (double)(1ull << nv[2]))};
        } else {
            figure_out_nv(nv, l);
        }
        const double voxel_size = 65536.0 * l;
        float3 lbf = LBF;
        if (origin == "center")
            lbf = float3{-(box.x / 2.0f), -(box.y / 2.0f), -(box.z / 2.0f)};
        else if (origin != "explicit")
            throw std::runtime_error("Unrecognized location of system origin.");
        if (bounding_bc != "none" && !bounding_added) {
            auto b = AddExternalObject();
            const float X = lbf.x, Y = lbf.y, Z = lbf.z, bx = box.x, by = box.y, bz = box.z;
            const auto& m = bounding_mat;
            b->AddPlane(float3{X + bx / 2.0f, Y + by / 2.0f, Z}, float3{0, 0, 1}, m);
            if (bounding_bc != "only_bottom") {
                b->AddPlane(float3{X, Y + by / 2.0f, Z + bz / 2.0f}, float3{1, 0, 0}, m);
                b->AddPlane(float3{X + bx, Y + by / 2.0f, Z + bz / 2.0f}, float3{-1, 0, 0}, m);
                b->AddPlane(float3{X + bx / 2.0f, Y, Z + bz / 2.0f}, float3{0, 1, 0}, m);
                b->AddPlane(float3{X + bx / 2.0f, Y + by, Z + bz / 2.0f}, float3{0, -1, 0}, m);
                if (bounding_bc != "top_open") b->AddPlane(float3{X + bx / 2.0f, Y + by / 2.0f, Z + bz}, float3{0, 0, -1}, m);
            }
            bounding_added = true;
        }
        std::vector<Presc> all_presc = presc;
        {  // validateUserInputs: the reserved family is fixed
            Presc p(DEME_RESERVED_FAMILY);
            p.linVel = {"0", "0", "0"};
            p.rotVel = {"0", "0", "0"};
            p.linVelP = p.rotVelP = p.linPosP = p.rotPosP = true;
            all_presc.push_back(p);
        }
        // ---- owners: clumps in batch order, then external objects, then mesh objects (dT.cpp:522-640,
        // kT.cpp:603-625) ----
        std::vector<const DEMClumpBatch*> bs;
        size_t nClumps = 0;
        for (const auto& b : batches) {
            bs.push_back(b.get());
            nClumps += b->nClumps;
        }
        const size_t nExt = ext.size(), nMesh = meshes.size(), nO = nClumps + nExt + nMesh;
        auto resize = [nO](auto&... v) { (v.resize(nO), ...); };
        resize(f.voxel, f.locX, f.locY, f.locZ, f.oriQw, f.oriQx, f.oriQy, f.oriQz, f.vX, f.vY, f.vZ, f.omgX, f.omgY,
               f.omgZ, f.family, f.mass, f.mmiXX, f.mmiYY, f.mmiZZ);
        std::vector<float3> pos(nO);
        size_t o = 0;
        f.template_names.clear();
        for (const auto& t : templates) f.template_names.push_back(t->m_name);
        for (const DEMClumpBatch* b : bs) {
            for (size_t i = 0; i < b->nClumps; i++, o++) {
                const DEMClumpTemplate& t = *b->types[i];
                pos[o] = b->xyz[i];
                f.oriQw[o] = b->oriQ[i].w;
                f.oriQx[o] = b->oriQ[i].x;
                f.oriQy[o] = b->oriQ[i].y;
                f.oriQz[o] = b->oriQ[i].z;
                f.vX[o] = b->vel[i].x;
                f.vY[o] = b->vel[i].y;
                f.vZ[o] = b->vel[i].z;
                f.omgX[o] = b->angVel[i].x;
                f.omgY[o] = b->angVel[i].y;
                f.omgZ[o] = b->angVel[i].z;
                f.family[o] = (uint8_t)b->families[i];
                f.mass[o] = t.mass;
                f.mmiXX[o] = t.MOI.x;
                f.mmiYY[o] = t.MOI.y;
                f.mmiZZ[o] = t.MOI.z;
                f.owner_template.push_back(t.mark);
                for (unsigned k = 0; k < t.nComp(); k++) {
                    f.sphere_owner.push_back((uint32_t)o);
                    f.radius.push_back(t.radii[k]);
                    f.relX.push_back(t.relPos[k].x);
                    f.relY.push_back(t.relPos[k].y);
                    f.relZ.push_back(t.relPos[k].z);
                    f.sphere_material.push_back((uint8_t)t.materials[k]->load_order);
                }
            }
        }
        for (size_t e = 0; e < nExt; e++, o++) {
            const DEMExternObj& x = *ext[e];
            pos[o] = x.init_pos;
            f.oriQw[o] = 1.f;
            f.oriQx[o] = f.oriQy[o] = f.oriQz[o] = 0.f;
            f.vX[o] = f.vY[o] = f.vZ[o] = f.omgX[o] = f.omgY[o] = f.omgZ[o] = 0.f;
            f.family[o] = (uint8_t)x.family_code;
            f.mass[o] = x.mass;
            f.mmiXX[o] = x.MOI.x;
            f.mmiYY[o] = x.MOI.y;
            f.mmiZZ[o] = x.MOI.z;
            for (const DEMAnalEntity& a : x.entities) {
                f.anal_type.push_back((uint8_t)a.type);
                f.anal_owner.push_back((uint32_t)o);
                f.anal_normal.push_back((uint8_t)a.normal);
                f.anal_material.push_back((uint8_t)a.material->load_order);
                f.anal_relX.push_back(a.pos.x);
                f.anal_relY.push_back(a.pos.y);
                f.anal_relZ.push_back(a.pos.z);
                f.anal_rotX.push_back(a.rot.x);
                f.anal_rotY.push_back(a.rot.y);
                f.anal_rotZ.push_back(a.rot.z);
                f.anal_size1.push_back(a.size1);
                f.anal_size2.push_back(a.size2);
                f.anal_size3.push_back(a.size3);
                f.anal_mass.push_back(x.mass);
            }
        }
        for (size_t e = 0; e < nMesh; e++, o++) {
            const DEMMeshConnected& x = *meshes[e];
            if (!x.isMaterialSet)
                throw std::runtime_error("A meshed object is loaded but does not have associated material. Please "
                                         "assign material to meshes via SetMaterial.");
            pos[o] = x.init_pos;
            f.oriQw[o] = x.init_oriQ.w;
            f.oriQx[o] = x.init_oriQ.x;
            f.oriQy[o] = x.init_oriQ.y;
            f.oriQz[o] = x.init_oriQ.z;
            f.vX[o] = x.init_vel.x;
            f.vY[o] = x.init_vel.y;
            f.vZ[o] = x.init_vel.z;
            f.omgX[o] = x.init_angvel.x;
            f.omgY[o] = x.init_angvel.y;
            f.omgZ[o] = x.init_angvel.z;
            f.family[o] = (uint8_t)x.family_code;
            f.mass[o] = x.mass;
            f.mmiXX[o] = x.MOI.x;
            f.mmiYY[o] = x.MOI.y;
            f.mmiZZ[o] = x.MOI.z;
            for (size_t i = 0; i < x.nTri; i++) {
                const std::array<float3, 3> t = x.FacetNodes(i);
                f.tri_owner.push_back((uint32_t)o);
                for (int c = 0; c < 3; c++) {
                    std::vector<float>* dst = c == 0 ? &f.tri_node1 : c == 1 ? &f.tri_node2 : &f.tri_node3;
                    dst->push_back(t[c].x);
                    dst->push_back(t[c].y);
                    dst->push_back(t[c].z);
                }
                f.tri_material.push_back((uint16_t)x.materials[i]->load_order);
            }
        }
        if (f.anal_type.size() > 255) throw std::runtime_error("at most 255 analytical components");
        // ---- initial encoding of xyz - LBF (hostPositionToVoxelID, HostSideHelpers.hpp:328-350) ----
        for (size_t i = 0; i < nO; i++) {
            uint16_t sub[3];
            encode_position(nv, voxel_size, l, (double)(pos[i].x - lbf.x), (double)(pos[i].y - lbf.y),
                            (double)(pos[i].z - lbf.z), f.voxel[i], sub);
            f.locX[i] = sub[0];
            f.locY[i] = sub[1];
            f.locZ[i] = sub[2];
        }
        // ---- materials ----
        auto prop = [](const DEMMaterial& m, const char* key) {
            auto it = m.mat_prop.find(key);
            return it == m.mat_prop.end() ? 0.f : it->second;
        };
        for (const auto& m : materials) {
            f.mat_E.push_back(prop(*m, "E"));
            f.mat_nu.push_back(prop(*m, "nu"));
            f.mat_CoR.push_back(prop(*m, "CoR"));
            f.mat_mu.push_back(prop(*m, "mu"));
            f.mat_Crr.push_back(prop(*m, "Crr"));
        }
        // ---- family masks and merged prescriptions (figureOutFamilyMasks, APIPrivate.cpp:574-645) ----
        f.family_masks.assign(DEME_NUM_FAMILY_MASK, 0);
        for (const auto& pr : no_contact) {
            const unsigned lo = std::min(pr.first, pr.second), hi = std::max(pr.first, pr.second);
            f.family_masks[(1 + hi) * hi / 2 + lo] = 1;
        }
        std::map<unsigned, Presc> merged;
        for (const Presc& p : all_presc) {
            auto it = merged.find(p.family);
            if (it == merged.end()) it = merged.emplace(p.family, Presc(p.family)).first;
            Presc& m = it->second;
            for (int k = 0; k < 3; k++) {
                if (p.linPos[k] != "none") m.linPos[k] = p.linPos[k];
                if (p.linVel[k] != "none") m.linVel[k] = p.linVel[k];
                if (p.rotVel[k] != "none") m.rotVel[k] = p.rotVel[k];
            }
            m.linVelP |= p.linVelP;
            m.rotVelP |= p.rotVelP;
            m.linPosP |= p.linPosP;
            m.rotPosP |= p.rotPosP;
        }
        f.prescriptions.assign(DEME_NUM_FAMILIES, deme_family_prescription{});
        f.motion_strings.clear();
        f.motion.clear();
        for (const auto& kv : merged) {
            deme_family_prescription& e = f.prescriptions[kv.first];
            const Presc& m = kv.second;
            bool expression = false;
            double v = 0.0;
            for (int k = 0; k < 3; k++)
                for (const std::string* x : {&m.linVel[k], &m.rotVel[k], &m.linPos[k]})
                    if (*x != "none" && !constant_expr(*x, v)) expression = true;
            if (expression) {  // the whole family goes to the compiled kernel; its table entry stays unused
                f.motion_strings.push_back({m.linVel[0], m.linVel[1], m.linVel[2], m.rotVel[0], m.rotVel[1],
                                            m.rotVel[2], m.linPos[0], m.linPos[1], m.linPos[2]});
                deme_motion_expressions me{};
                me.family = (int32_t)kv.first;
                me.lin_vel_prescribed = m.linVelP;
                me.rot_vel_prescribed = m.rotVelP;
                me.lin_pos_prescribed = m.linPosP;
                me.rot_pos_prescribed = m.rotPosP;
                f.motion.push_back(me);
                continue;
            }
            e.used = 1;
            e.lin_vel_prescribed = m.linVelP;
            e.rot_vel_prescribed = m.rotVelP;
            e.lin_pos_prescribed = m.linPosP;
            e.rot_pos_prescribed = m.rotPosP;
            for (int k = 0; k < 3; k++) {
                if (m.linVel[k] != "none" && constant_expr(m.linVel[k], v)) {
                    e.has_vel[k] = 1;
                    e.vel[k] = (float)v;
                }
                if (m.rotVel[k] != "none" && constant_expr(m.rotVel[k], v)) {
                    e.has_omg[k] = 1;
                    e.omg[k] = (float)v;
                }
                if (m.linPos[k] != "none" && constant_expr(m.linPos[k], v)) {
                    e.has_pos[k] = 1;
                    e.pos[k] = v;
                }
            }
        }
        // ---- bins (decideBinSize, APIPrivate.cpp:335-369) and expand factor (APIPrivate.cpp:730-758) ----
        double rmin = HUGE_VAL;
        for (float r : f.radius) rmin = std::min(rmin, (double)r);
        for (const auto& t : templates)
            for (float r : t->radii) rmin = std::min(rmin, (double)r);
        double bs_ = bin_size;
        if (!(bs_ > 0.0)) {
            if (!(rmin > 1e-12)) throw std::runtime_error("spheres with zero radius and no bin size given");
            bs_ = 2.0 * (double)(float)rmin;
        }
        uint32_t nb[3];
        for (int i = 0; i < 3; i++) nb[i] = (uint32_t)(voxel_size * std::ldexp(1.0, nv[i]) / bs_) + 1u;
        const double beta = expand_fixed ? (double)expand_factor
                                         : (double)(float)((double)max_vel * h_step * update_freq * (double)safety);
        deme_sim_params& p = f.params;
        p = deme_sim_params{};
        p.nvXp2 = nv[0];
        p.nvYp2 = nv[1];
        p.nvZp2 = nv[2];
        p.nbX = nb[0];
        p.nbY = nb[1];
        p.nbZ = nb[2];
        p.l = l;
        p.voxel_size = voxel_size;
        p.l_kernel = kernel_literal(l);
        p.voxel_size_kernel = kernel_literal(voxel_size);
        p.bin_size = bs_;
        p.lbf[0] = lbf.x;
        p.lbf[1] = lbf.y;
        p.lbf[2] = lbf.z;
        p.G[0] = G.x;
        p.G[1] = G.y;
        p.G[2] = G.z;
        p.h = (float)h_step;
        p.beta = (float)beta;
        p.integrator = integrator;
        p.cd_update_freq = update_freq;
        p.n_contact_wildcards = force_model && force_model->custom ? (int32_t)force_model->m_contact_wildcards.size()
                                : (force_model && force_model->frictionless ? 0 : 4);
        p.domain[0] = box.x;
        p.domain[1] = box.y;
        p.domain[2] = box.z;
        f.point();
    }

    std::vector<std::shared_ptr<DEMMaterial>> materials;
    std::vector<std::shared_ptr<DEMClumpTemplate>> templates;
    std::vector<std::shared_ptr<DEMClumpBatch>> batches;
    std::vector<std::shared_ptr<DEMExternObj>> ext;
    std::vector<std::shared_ptr<DEMMeshConnected>> meshes;
    float3 box{0.f, 0.f, 0.f};
    bool has_box = false;
    bool has_explicit_nv = false;  // InstructBoxDomainNumVoxel
    bool timing_on = false;        // EnableTimingStats
    uint8_t explicit_nv[3] = {0, 0, 0};
    float explicit_l = 0.f;
    std::string origin = "explicit";
    float3 LBF{0.f, 0.f, 0.f};
    std::string bounding_bc = "none";
    std::shared_ptr<DEMMaterial> bounding_mat;
    bool bounding_added = false;
    float3 G{0.f, 0.f, 0.f};
    double h_step = -1.0;
    double bin_size = -1.0;
    float expand_factor = 0.f;
    bool expand_fixed = false;
    float max_vel = -1.f;
    float safety = 1.f;
    int update_freq = 0;
    int integrator = DEME_INTEGRATOR_EXTENDED_TAYLOR;
    std::vector<std::pair<unsigned, unsigned>> no_contact;
    std::vector<Presc> presc;
    std::shared_ptr<DEMForceModel> force_model;
    std::unique_ptr<FlatScene> flat;
    deme_handle* h = nullptr;
    struct FamilyRule {
        unsigned from, to;
        std::string condition;
    };
    std::vector<FamilyRule> fam_rules;
    unsigned out_content = OUTPUT_CONTENT::QUAT | OUTPUT_CONTENT::ABSV;
    unsigned cnt_out_content = CNT_OUTPUT_CONTENT::FORCE | CNT_OUTPUT_CONTENT::POINT;
    std::set<unsigned> no_output;
    // the system's clump batches (flattened into the handle, in order) and what UpdateClumps checks against
    std::vector<std::shared_ptr<DEMClumpBatch>> system_batches;
    size_t n_clumps_init = 0, n_clumps_system = 0, n_ext_init = 0, n_mesh_init = 0, n_templates_init = 0,
           n_materials_init = 0, n_presc_init = 0;
};

inline float DEMInspector::GetValue() { return sys->InspectValue(quantity); }
inline uint32_t DEMTracker::OwnerID() { return sys->TrackedOwnerID(obj, kind); }
inline float3 DEMTracker::Pos(size_t offset) { return sys->GetOwnerPosition(OwnerID() + (uint32_t)offset); }
inline float3 DEMTracker::AngVelLocal(size_t offset) { return sys->GetOwnerAngVel(OwnerID() + (uint32_t)offset); }
inline float3 DEMTracker::Vel(size_t offset) { return sys->GetOwnerVelocity(OwnerID() + (uint32_t)offset); }
inline float4 DEMTracker::OriQ(size_t offset) { return sys->GetOwnerOriQ(OwnerID() + (uint32_t)offset); }
inline float3 DEMTracker::ContactAcc(size_t offset) { return sys->GetOwnerAcc(OwnerID() + (uint32_t)offset); }
inline float3 DEMTracker::ContactAngAccLocal(size_t offset) {
    return sys->GetOwnerAngAcc(OwnerID() + (uint32_t)offset);
}
inline void DEMTracker::SetPos(float3 pos, size_t offset) {
    sys->SetOwnerPosition(OwnerID() + (uint32_t)offset, pos);
}
inline void DEMTracker::SetAngVel(float3 w, size_t offset) { sys->SetOwnerAngVel(OwnerID() + (uint32_t)offset, w); }
inline void DEMTracker::SetVel(float3 v, size_t offset) { sys->SetOwnerVelocity(OwnerID() + (uint32_t)offset, v); }
inline void DEMTracker::SetOriQ(float4 q, size_t offset) { sys->SetOwnerOriQ(OwnerID() + (uint32_t)offset, q); }
inline void DEMTracker::ChangeClumpSizes(const std::vector<uint32_t>& ids, const std::vector<float>& factors) {
    std::vector<uint32_t> shifted(ids);
    const uint32_t first = OwnerID();
    for (auto& x : shifted) x += first;
    sys->ChangeClumpSizes(shifted, factors);
}

}  // namespace deme

#endif /* DEME_SOLVER_HPP */
