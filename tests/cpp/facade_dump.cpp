// Builds one scene through the C++ DEMSolver facade (include/deme_solver.hpp) from per-clump inputs written by
// tests/test_cpp_facade.py, flattens it (no GPU needed) and writes every flat array for comparison with the Python
// SceneBuilder.  With a step count it also initializes the solver on the GPU, steps, and writes the owner state.
// With "ops" after the step count it then exercises the per-owner setters and getters (SetOwner* / GetOwnerAcc /
// GetOwnerAngAcc) and UpdateClumps, writing what it set and what it read back.
// Usage: facade_dump <inputs.bin> <out.bin> [steps [ops]]
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>

#include "deme_solver.hpp"

using namespace deme;

template <typename T>
static std::vector<T> read_vec(std::ifstream& in) {
    uint64_t n = 0;
    in.read(reinterpret_cast<char*>(&n), sizeof(n));
    std::vector<T> v(n);
    in.read(reinterpret_cast<char*>(v.data()), (std::streamsize)(n * sizeof(T)));
    return v;
}

template <typename T>
static void put(std::ofstream& out, const char* name, const T* data, size_t n) {
    const uint32_t len = (uint32_t)std::strlen(name);
    const uint64_t bytes = n * sizeof(T);
    out.write(reinterpret_cast<const char*>(&len), sizeof(len));
    out.write(name, len);
    out.write(reinterpret_cast<const char*>(&bytes), sizeof(bytes));
    out.write(reinterpret_cast<const char*>(data), (std::streamsize)bytes);
}
template <typename T>
static void put(std::ofstream& out, const char* name, const std::vector<T>& v) {
    put(out, name, v.data(), v.size());
}

// the mesh body of the scene (the Python side writes the same text)
static const char* kMeshObj =
    "v 0 0 0\nv 0.02 0 0\nv 0.02 0.02 0\nv 0 0.02 0\nv 0.01 0.01 0.015\n"
    "f 1 2 3 4\nf 1/1 2/1 5/1\nf -4 -3 -1\nf 3 4 5\nf 4 1 5\n";

// the third clump template's components (the Python side writes the same text)
static const char* kClumpCsv = "r,note,x,y,z\n0.004,top,0,0,0.0025\n0.004,bottom,0,0,-0.0025\n";

int main(int argc, char** argv) {
    if (argc < 3 || argc > 5) return 2;
    std::ifstream in(argv[1], std::ios::binary);
    const auto types = read_vec<int32_t>(in);    // batch 1 template index per clump
    const auto xyz1 = read_vec<float>(in);       // batch 1 positions (3 per clump)
    const auto q1 = read_vec<float>(in);         // batch 1 quaternions (w, x, y, z)
    const auto v1 = read_vec<float>(in);         // batch 1 velocities
    const auto w1 = read_vec<float>(in);         // batch 1 angular velocities
    const auto fam1 = read_vec<int32_t>(in);     // batch 1 families
    const auto xyz2 = read_vec<float>(in);       // batch 2 positions

    DEMSolver s;
    std::vector<float> mesh_props;
    const bool numvoxel = argc >= 4 && std::string(argv[3]) == "nv";
    if (numvoxel)
        s.InstructBoxDomainNumVoxel(21, 21, 22, 4e-12f);
    else
        s.InstructBoxDomainDimension(0.3f, 0.3f, 0.45f);
    // switches of the reference that have no effect here must still compile
    s.SetVerbosity(INFO);
    s.SetOutputFormat(OUTPUT_FORMAT::CSV);
    s.SetSortContactPairs(true);
    s.InstructNumOwners(100);
    s.SetFamilyPrescribedQuaternion(4, "none");
    s.PurgeFamily(4);
    s.SetCoordSysOrigin("center");
    auto m0 = s.LoadMaterial({{"E", 1e7f}, {"nu", 0.3f}, {"CoR", 0.5f}, {"mu", 0.5f}, {"Crr", 0.0f}});
    auto m1 = s.LoadMaterial({{"E", 5e7f}, {"nu", 0.25f}, {"CoR", 0.3f}, {"mu", 0.4f}, {"Crr", 0.02f}});
    s.InstructBoxDomainBoundingBC("top_open", m0);
    std::vector<std::shared_ptr<DEMClumpTemplate>> T;
    T.push_back(s.LoadSphereType(1.361e-3f, 5e-3f, m0));
    T.push_back(s.LoadClumpType(2.5e-3f, float3{1e-7f, 1.2e-7f, 1.5e-7f}, {4e-3f, 5e-3f, 4.5e-3f},
                                {float3{3e-3f, 0.f, 0.f}, float3{-1.5e-3f, 2.6e-3f, 0.f}, float3{-1.5e-3f, -2.6e-3f, 0.f}},
                                {m0, m1, m0}));
    {
        // the third template from a clump file (header names the columns; an extra column is ignored)
        const std::string csv = std::string(argv[2]) + ".clump.csv";
        std::ofstream(csv) << kClumpCsv;
        T.push_back(s.LoadClumpType(1.8e-3f, float3{8e-8f, 9e-8f, 9e-8f}, csv, m1));
    }
    const size_t n1 = types.size(), n2 = xyz2.size() / 3;
    std::vector<std::shared_ptr<DEMClumpTemplate>> tv;
    std::vector<float3> p1, vv, ww, p2;
    std::vector<float4> qq;
    std::vector<unsigned> ff;
    for (size_t i = 0; i < n1; i++) {
        tv.push_back(T[types[i]]);
        p1.push_back(float3{xyz1[3 * i], xyz1[3 * i + 1], xyz1[3 * i + 2]});
        qq.push_back(float4{q1[4 * i + 1], q1[4 * i + 2], q1[4 * i + 3], q1[4 * i]});
        vv.push_back(float3{v1[3 * i], v1[3 * i + 1], v1[3 * i + 2]});
        ww.push_back(float3{w1[3 * i], w1[3 * i + 1], w1[3 * i + 2]});
        ff.push_back((unsigned)fam1[i]);
    }
    for (size_t i = 0; i < n2; i++) p2.push_back(float3{xyz2[3 * i], xyz2[3 * i + 1], xyz2[3 * i + 2]});
    auto b1 = s.AddClumps(tv, p1);
    b1->SetOriQ(qq);
    b1->SetVel(vv);
    b1->SetAngVel(ww);
    b1->SetFamilies(ff);
    auto b2 = s.AddClumps(T[2], p2);
    b2->SetFamily(3);
    s.AddBCPlane(float3{0.f, 0.f, -0.1f}, float3{0.1f, 0.f, 1.f}, m1);
    auto wall = s.AddExternalObject();
    wall->AddCylinder(float3{0.f, 0.f, 0.f}, float3{0.f, 0.f, 1.f}, 0.12f, m0);
    wall->AddPlate(float3{0.f, 0.05f, -0.15f}, float3{0.f, 0.f, 1.f}, 0.04f, 0.03f, m0);
    wall->AddCone(float3{0.f, 0.f, -0.2f}, float3{0.f, 0.f, 1.f}, 0.5235988f, 0.03f, 0.15f, m1);
    wall->SetFamily(10);
    {
        // a mesh body (Wavefront file, a quad split in two and four triangles, per-facet materials)
        const std::string obj = std::string(argv[2]) + ".obj";
        std::ofstream(obj) << kMeshObj;
        auto mesh = s.AddWavefrontMeshObject(obj, m0);
        mesh->SetMaterial(std::vector<std::shared_ptr<DEMMaterial>>{m0, m1, m0, m1, m0, m1});
        mesh->SetInitPos(float3{0.02f, 0.08f, -0.06f});
        mesh->SetInitQuat(float4{0.f, 0.6f, 0.f, 0.8f});
        mesh->SetMass(2.5f);
        mesh->SetMOI(float3{1e-3f, 2e-3f, 3e-3f});
        mesh->SetFamily(3);
        // mesh utilities: a rotated copy's mass properties, and both written back as one Wavefront file
        DEMMeshConnected copy(obj);
        copy.Rotate(float4{0.f, 0.6f, 0.f, 0.8f});
        double mp_mass = 0.0;
        float3 mp_c{0.f, 0.f, 0.f}, mp_i{0.f, 0.f, 0.f};
        copy.ComputeMassProperties(mp_mass, mp_c, mp_i);
        mesh_props = {(float)mp_mass, mp_c.x, mp_c.y, mp_c.z, mp_i.x, mp_i.y, mp_i.z};
        std::vector<DEMMeshConnected> both{*mesh, copy};
        DEMMeshConnected::WriteWavefront(std::string(argv[2]) + ".out.obj", both);
    }
    s.SetFamilyFixed(3);
    s.SetFamilyPrescribedAngVel(10, "0", "2.0943951", "0");
    s.SetFamilyPrescribedLinVel(4, "0.1", "none", "0");
    s.SetFamilyPrescribedLinVel(5, "0", "0", "0.2 * sin(3000.0 * t)");
    s.DisableContactBetweenFamilies(3, 10);
    s.SetInitTimeStep(1e-5);
    s.SetGravitationalAcceleration(float3{0.f, 0.f, -9.81f});
    s.SetCDUpdateFreq(5);
    s.SetExpandFactor(1e-4f);
    const FlatScene& f = s.Flatten();

    std::ofstream out(argv[2], std::ios::binary);
    put(out, "params", &f.params, 1);
    put(out, "voxel", f.voxel);
    put(out, "locX", f.locX);
    put(out, "locY", f.locY);
    put(out, "locZ", f.locZ);
    put(out, "oriQw", f.oriQw);
    put(out, "oriQx", f.oriQx);
    put(out, "oriQy", f.oriQy);
    put(out, "oriQz", f.oriQz);
    put(out, "vX", f.vX);
    put(out, "vY", f.vY);
    put(out, "vZ", f.vZ);
    put(out, "omgX", f.omgX);
    put(out, "omgY", f.omgY);
    put(out, "omgZ", f.omgZ);
    put(out, "family", f.family);
    put(out, "mass", f.mass);
    put(out, "mmiXX", f.mmiXX);
    put(out, "mmiYY", f.mmiYY);
    put(out, "mmiZZ", f.mmiZZ);
    put(out, "sphere_owner", f.sphere_owner);
    put(out, "relX", f.relX);
    put(out, "relY", f.relY);
    put(out, "relZ", f.relZ);
    put(out, "radius", f.radius);
    put(out, "sphere_material", f.sphere_material);
    put(out, "anal_type", f.anal_type);
    put(out, "anal_owner", f.anal_owner);
    put(out, "anal_normal", f.anal_normal);
    put(out, "anal_material", f.anal_material);
    put(out, "anal_relX", f.anal_relX);
    put(out, "anal_relY", f.anal_relY);
    put(out, "anal_relZ", f.anal_relZ);
    put(out, "anal_rotX", f.anal_rotX);
    put(out, "anal_rotY", f.anal_rotY);
    put(out, "anal_rotZ", f.anal_rotZ);
    put(out, "anal_size1", f.anal_size1);
    put(out, "anal_size2", f.anal_size2);
    put(out, "anal_size3", f.anal_size3);
    put(out, "anal_mass", f.anal_mass);
    put(out, "mat_E", f.mat_E);
    put(out, "mat_nu", f.mat_nu);
    put(out, "mat_CoR", f.mat_CoR);
    put(out, "mat_mu", f.mat_mu);
    put(out, "mat_Crr", f.mat_Crr);
    put(out, "family_masks", f.family_masks);
    put(out, "mesh_props", mesh_props);
    put(out, "tri_owner", f.tri_owner);
    put(out, "tri_node1", f.tri_node1);
    put(out, "tri_node2", f.tri_node2);
    put(out, "tri_node3", f.tri_node3);
    put(out, "tri_material", f.tri_material);
    put(out, "prescriptions", f.prescriptions);
    {
        // families handed to deme_set_prescribed_motion: family, four flags, nine strings, '|'-separated lines
        std::string m;
        for (size_t i = 0; i < f.motion.size(); i++) {
            const deme_motion_expressions& e = f.motion[i];
            m += std::to_string(e.family) + "|" + std::to_string(e.lin_vel_prescribed) + "|" +
                 std::to_string(e.rot_vel_prescribed) + "|" + std::to_string(e.lin_pos_prescribed) + "|" +
                 std::to_string(e.rot_pos_prescribed);
            for (const std::string& x : f.motion_strings[i]) m += "|" + x;
            m += "\n";
        }
        put(out, "motion", m.data(), m.size());
    }
    {
        // CSV output of the initial state (every column), for comparison with the Python writers
        OwnerState st;
        st.voxel = f.voxel;
        st.locX = f.locX;
        st.locY = f.locY;
        st.locZ = f.locZ;
        st.oriQw = f.oriQw;
        st.oriQx = f.oriQx;
        st.oriQy = f.oriQy;
        st.oriQz = f.oriQz;
        st.vX = f.vX;
        st.vY = f.vY;
        st.vZ = f.vZ;
        st.family = f.family;
        st.omgX = f.omgX;
        st.omgY = f.omgY;
        st.omgZ = f.omgZ;
        {
            // the inspectors' reductions on the initial state (template volumes 1, 2, 3)
            const float insp[4] = {inspect_quantity(f, st, "clump_max_z", {1.f, 2.f, 3.f}),
                                   inspect_quantity(f, st, "clump_min_z", {1.f, 2.f, 3.f}),
                                   inspect_quantity(f, st, "clump_max_absv", {1.f, 2.f, 3.f}),
                                   inspect_quantity(f, st, "clump_volume", {1.f, 2.f, 3.f})};
            put(out, "inspect", insp, 4);
        }
        const unsigned all = OUTPUT_CONTENT::ABSV | OUTPUT_CONTENT::VEL | OUTPUT_CONTENT::FAMILY;
        std::ostringstream sph, clu;
        write_sphere_csv(sph, f, st, all, {3});
        write_clump_csv(clu, f, st, all);
        const std::string a = sph.str(), b = clu.str();
        put(out, "csv_spheres", a.data(), a.size());
        put(out, "csv_clumps", b.data(), b.size());
        // a contact file from a synthetic list: two sphere pairs and one sphere--plane contact
        const std::vector<uint32_t> idA{0, 1, 2}, idB{1, 3, 0};
        const std::vector<uint8_t> type{DEME_SPHERE_SPHERE_CONTACT, DEME_SPHERE_SPHERE_CONTACT,
                                        DEME_SPHERE_PLANE_CONTACT};
        std::vector<float> F(9), T(9), P(9);
        for (int i = 0; i < 9; i++) {
            F[i] = 0.5f * (float)(i + 1) - 1.25f;
            T[i] = 0.01f * (float)(i * i);
            P[i] = 1e-3f * (float)(i % 3 + 1) * (i % 2 ? -1.f : 1.f);
        }
        std::ostringstream cnt;
        write_contact_csv(cnt, f, st, idA, idB, type, F, T, P,
                          CNT_OUTPUT_CONTENT::FORCE | CNT_OUTPUT_CONTENT::POINT | CNT_OUTPUT_CONTENT::NORMAL |
                              CNT_OUTPUT_CONTENT::TORQUE_ONLY_FORCE);
        const std::string c = cnt.str();
        put(out, "csv_contacts", c.data(), c.size());
    }
    if (argc >= 4 && !numvoxel) {
        const int steps = std::atoi(argv[3]);
        s.Initialize();  // flattens again: use the new FlatScene from here on
        for (int i = 0; i < steps; i++) s.DoStepDynamics();
        const size_t nO = s.GetFlatScene().voxel.size();
        std::vector<float3> pos(nO), vel(nO);
        for (size_t o = 0; o < nO; o++) {
            pos[o] = s.GetOwnerPosition((uint32_t)o);
            vel[o] = s.GetOwnerVelocity((uint32_t)o);
        }
        const double ke = s.GetTotalKineticEnergy();
        const uint32_t nc = s.GetNumContacts();
        put(out, "run_pos", pos);
        put(out, "run_vel", vel);
        put(out, "run_ke", &ke, 1);
        put(out, "run_ncontacts", &nc, 1);
        if (argc == 5 && std::string(argv[4]) == "ops") {
            // accelerations of the last step, owner by owner
            std::vector<float3> acc(nO), aacc(nO);
            for (size_t o = 0; o < nO; o++) {
                acc[o] = s.GetOwnerAcc((uint32_t)o);
                aacc[o] = s.GetOwnerAngAcc((uint32_t)o);
            }
            put(out, "ops_acc", acc);
            put(out, "ops_angacc", aacc);
            // one setter per owner 0..3, read back, then one more step
            const float3 p0{0.01f, -0.02f, 0.05f}, v1{0.3f, -0.1f, 0.2f}, w2{5.f, -3.f, 1.f};
            const float4 q3{0.f, 0.6f, 0.f, 0.8f};  // (x, y, z, w)
            s.SetOwnerPosition(0, p0);
            s.SetOwnerVelocity(1, v1);
            s.SetOwnerAngVel(2, w2);
            s.SetOwnerOriQ(3, q3);
            const float3 rb[3] = {s.GetOwnerPosition(0), s.GetOwnerVelocity(1), s.GetOwnerAngVel(2)};
            const float4 rq = s.GetOwnerOriQ(3);
            put(out, "ops_readback", rb, 3);
            put(out, "ops_readback_q", &rq, 1);
            s.DoStepDynamics();
            for (size_t o = 0; o < nO; o++) {
                pos[o] = s.GetOwnerPosition((uint32_t)o);
                vel[o] = s.GetOwnerVelocity((uint32_t)o);
            }
            put(out, "ops_pos", pos);
            put(out, "ops_vel", vel);
            // trackers of the second batch (its first clump and the next) and of the cylinder-and-cone object
            auto t2 = s.Track(b2);
            auto tw = s.Track(wall);
            const float3 tr[3] = {t2->Pos(0), t2->Vel(1), tw->Pos()};
            const uint32_t tid[2] = {t2->OwnerID(), tw->OwnerID()};
            put(out, "trk", tr, 3);
            put(out, "trk_id", tid, 2);
            // UpdateClumps: forget the cached batches, add three spheres, carry the run over
            const uint32_t nc_before = s.GetNumContacts();
            const double t_before = s.GetSimTime();
            s.ClearCache();
            std::vector<float3> p3{float3{-0.05f, 0.05f, 0.15f}, float3{0.05f, 0.05f, 0.15f},
                                   float3{0.f, -0.05f, 0.15f}};
            auto b3 = s.AddClumps(T[0], p3);
            b3->SetVel(std::vector<float3>(3, float3{0.f, 0.f, -0.5f}));
            s.UpdateClumps();
            const size_t nO2 = s.GetFlatScene().voxel.size();
            std::vector<float3> upos(nO2), uvel(nO2);
            for (size_t o = 0; o < nO2; o++) {
                upos[o] = s.GetOwnerPosition((uint32_t)o);
                uvel[o] = s.GetOwnerVelocity((uint32_t)o);
            }
            const uint32_t nc_after = s.GetNumContacts();
            const double t_after = s.GetSimTime();
            put(out, "upd_pos", upos);
            put(out, "upd_vel", uvel);
            const uint32_t ncs[2] = {nc_before, nc_after};
            const double ts[2] = {t_before, t_after};
            put(out, "upd_ncontacts", ncs, 2);
            put(out, "upd_time", ts, 2);
            for (int i = 0; i < 3; i++) s.DoStepDynamics();
            for (size_t o = 0; o < nO2; o++) upos[o] = s.GetOwnerPosition((uint32_t)o);
            put(out, "upd_pos_after", upos);
        }
    }
    return 0;
}
