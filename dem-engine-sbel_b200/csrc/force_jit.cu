// force_jit.cu -- compiles a DEM-Engine force-model string into the force kernel with NVRTC.
//
// The reference pastes the model string into its jitified force kernel (src/DEM/APIPrivate.cpp:925-978 with the
// ingredient and wildcard code of src/DEM/Models.h:197-256).  Here the string goes into this project's own kernel
// template, force_kernel.cuh, the same source the built-in model is compiled from: NVRTC receives that header set
// (embedded in the library at build time) plus one generated file holding the wildcard loads, the model, and the
// wildcard stores.  The result is loaded as a CUDA library and launched through the runtime API.
#include <algorithm>
#include <cctype>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include <nvrtc.h>

#include "../../include/deme_b200.h"
#include "force_jit.cuh"

namespace deme_b200 {
namespace {

struct JitHeader {
    const char* name;
    const char* text;
};

// force_kernel.cuh and the headers it includes, embedded by the build (see the Makefile rule for jit_sources.inc)
const JitHeader kJitHeaders[] = {
#include "jit_sources.inc"
};

const char* kStdintStub =
    "#pragma once\n"
    "typedef signed char int8_t; typedef short int16_t; typedef int int32_t; typedef long long int64_t;\n"
    "typedef unsigned char uint8_t; typedef unsigned short uint16_t; typedef unsigned int uint32_t;\n"
    "typedef unsigned long long uint64_t; typedef unsigned long long uintptr_t;\n";
const char* kStddefStub = "#pragma once\ntypedef unsigned long size_t;\n";

const char* kMainSource =
    "#define DEME_USER_FORCE_MODEL 1\n"
    "#include <stdint.h>\n"
    "#include \"force_model_api.cuh\"\n"
    "#include \"force_kernel.cuh\"\n";

bool is_identifier(const char* s) {
    if (!s || !*s || !(std::isalpha((unsigned char)s[0]) || s[0] == '_')) return false;
    for (const char* p = s; *p; p++)
        if (!(std::isalnum((unsigned char)*p) || *p == '_')) return false;
    return true;
}

// Compiled images by (architecture, generated model text): re-declaring the same model skips NVRTC.
struct CompiledModel {
    std::vector<char> cubin;
    std::string lowered[2];
};
std::mutex g_cache_mutex;
std::unordered_map<std::string, CompiledModel> g_cache;

}  // namespace

int32_t compile_user_force_model(const char* model, const char* const* names, int32_t n, UserForceKernel& out,
                                 std::string& err) {
    if (!model) {
        err = "force model string is null";
        return DEME_ERR_INVALID;
    }
    if (n < 0 || n > kMaxContactWildcards) {
        err = "a force model may declare at most " + std::to_string(kMaxContactWildcards) + " contact wildcards";
        return DEME_ERR_INVALID;
    }
    std::vector<std::string> wc;
    for (int32_t i = 0; i < n; i++) {
        if (!is_identifier(names ? names[i] : nullptr)) {
            err = "contact wildcard name " + std::to_string(i) + " is not an identifier";
            return DEME_ERR_INVALID;
        }
        wc.emplace_back(names[i]);
    }
    std::sort(wc.begin(), wc.end());
    if (std::adjacent_find(wc.begin(), wc.end()) != wc.end()) {
        err = "duplicate contact wildcard name";
        return DEME_ERR_INVALID;
    }
    // contact wildcards in, the model, contact wildcards out (equip_contact_wildcards, src/DEM/Models.h:237-256)
    static const char* kSlots[kMaxContactWildcards] = {"hw.x", "hw.y", "hw.z", "hw.w"};
    std::string inc;
    for (size_t i = 0; i < wc.size(); i++) inc += "float " + wc[i] + " = " + kSlots[i] + ";\n";
    inc += "{\n#line 1 \"force_model_string\"\n";
    inc += model;
    inc += "\n}\n";
    for (size_t i = 0; i < wc.size(); i++) inc += std::string(kSlots[i]) + " = " + wc[i] + ";\n";

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        err = "no current CUDA device";
        return DEME_ERR_NO_DEVICE;
    }
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
        err = "cudaGetDeviceProperties failed";
        return DEME_ERR_CUDA;
    }
    const std::string arch = "--gpu-architecture=sm_" + std::to_string(prop.major * 10 + prop.minor) +
                             (prop.major >= 9 ? "a" : "");
    const std::string key = arch + "\n" + inc;

    CompiledModel cm;
    bool cached = false;
    {
        std::lock_guard<std::mutex> lock(g_cache_mutex);
        auto it = g_cache.find(key);
        if (it != g_cache.end()) {
            cm = it->second;
            cached = true;
        }
    }
    if (!cached) {
        const char* exprs[2] = {"deme_b200::k_force<false>", "deme_b200::k_force<true>"};
        std::vector<const char*> hnames, htexts;
        for (const JitHeader& hdr : kJitHeaders) {
            hnames.push_back(hdr.name);
            htexts.push_back(hdr.text);
        }
        hnames.push_back("stdint.h");
        htexts.push_back(kStdintStub);
        hnames.push_back("stddef.h");
        htexts.push_back(kStddefStub);
        hnames.push_back("deme_user_force_model.inc");
        htexts.push_back(inc.c_str());
        nvrtcProgram prog = nullptr;
        if (nvrtcCreateProgram(&prog, kMainSource, "deme_user_force.cu", (int)hnames.size(), htexts.data(),
                               hnames.data()) != NVRTC_SUCCESS) {
            err = "nvrtcCreateProgram failed";
            return DEME_ERR_NVRTC;
        }
        for (const char* e : exprs) nvrtcAddNameExpression(prog, e);
        const char* opts[] = {arch.c_str(), "--fmad=false", "-std=c++17", "-lineinfo"};
        const nvrtcResult rc = nvrtcCompileProgram(prog, 4, opts);
        if (rc != NVRTC_SUCCESS) {
            size_t logSize = 0;
            nvrtcGetProgramLogSize(prog, &logSize);
            std::string log(logSize, '\0');
            if (logSize) nvrtcGetProgramLog(prog, &log[0]);
            err = std::string("force model did not compile: ") + nvrtcGetErrorString(rc) + "\n" + log;
            nvrtcDestroyProgram(&prog);
            return DEME_ERR_NVRTC;
        }
        size_t sz = 0;
        bool ok = nvrtcGetCUBINSize(prog, &sz) == NVRTC_SUCCESS && sz > 0;
        if (ok) {
            cm.cubin.resize(sz);
            ok = nvrtcGetCUBIN(prog, cm.cubin.data()) == NVRTC_SUCCESS;
        }
        for (int i = 0; ok && i < 2; i++) {
            const char* name = nullptr;
            ok = nvrtcGetLoweredName(prog, exprs[i], &name) == NVRTC_SUCCESS && name;
            if (ok) cm.lowered[i] = name;
        }
        nvrtcDestroyProgram(&prog);
        if (!ok) {
            err = "NVRTC produced no loadable image for the force model";
            return DEME_ERR_NVRTC;
        }
        std::lock_guard<std::mutex> lock(g_cache_mutex);
        g_cache[key] = cm;
    }

    UserForceKernel k;
    if (cudaLibraryLoadData(&k.lib, cm.cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0) != cudaSuccess) {
        err = std::string("loading the compiled force model failed: ") + cudaGetErrorString(cudaGetLastError());
        return DEME_ERR_CUDA;
    }
    for (int i = 0; i < 2; i++) {
        if (cudaLibraryGetKernel(&k.kern[i], k.lib, cm.lowered[i].c_str()) != cudaSuccess) {
            err = "compiled force model lacks its kernel";
            cudaLibraryUnload(k.lib);
            return DEME_ERR_CUDA;
        }
    }
    k.n_wildcards = (int)wc.size();
    release_user_force_model(out);
    out = k;
    return DEME_OK;
}

void release_user_force_model(UserForceKernel& k) {
    if (k.lib) cudaLibraryUnload(k.lib);
    k = UserForceKernel{};
}

namespace {
// Every whole-word `return` of a condition becomes `shouldMakeChange =` (the reference's replace_pattern).
std::string returns_to_decision(const std::string& c) {
    std::string out;
    size_t i = 0;
    auto word = [](char ch) { return std::isalnum((unsigned char)ch) || ch == '_'; };
    while (i < c.size()) {
        if (c.compare(i, 6, "return") == 0 && (i == 0 || !word(c[i - 1])) && (i + 6 >= c.size() || !word(c[i + 6]))) {
            out += "shouldMakeChange =";
            i += 6;
        } else {
            out += c[i++];
        }
    }
    return out;
}

const char* kFamilySource =
    "#include <stdint.h>\n"
    "#include \"force_model_api.cuh\"\n"
    "#include \"family_change_kernel.cuh\"\n";
}  // namespace

namespace {

// Compiles `source` for the current device with the embedded header set plus the generated files `extra`
// (name, text), and loads the kernel named by `expr`.  `what` names the user input in error messages.
int32_t build_one_kernel(const char* source, const char* prog_name,
                         const std::vector<std::pair<std::string, std::string>>& extra, const char* expr,
                         const char* what, cudaLibrary_t& lib, cudaKernel_t& kern, std::string& err) {
    int dev = 0;
    cudaDeviceProp prop{};
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
        err = "no current CUDA device";
        return DEME_ERR_NO_DEVICE;
    }
    const std::string arch = "--gpu-architecture=sm_" + std::to_string(prop.major * 10 + prop.minor) +
                             (prop.major >= 9 ? "a" : "");
    std::vector<const char*> hnames, htexts;
    for (const JitHeader& hdr : kJitHeaders) {
        hnames.push_back(hdr.name);
        htexts.push_back(hdr.text);
    }
    hnames.push_back("stdint.h");
    htexts.push_back(kStdintStub);
    hnames.push_back("stddef.h");
    htexts.push_back(kStddefStub);
    for (const auto& e : extra) {
        hnames.push_back(e.first.c_str());
        htexts.push_back(e.second.c_str());
    }
    nvrtcProgram prog = nullptr;
    if (nvrtcCreateProgram(&prog, source, prog_name, (int)hnames.size(), htexts.data(), hnames.data()) !=
        NVRTC_SUCCESS) {
        err = "nvrtcCreateProgram failed";
        return DEME_ERR_NVRTC;
    }
    nvrtcAddNameExpression(prog, expr);
    const char* opts[] = {arch.c_str(), "--fmad=false", "-std=c++17", "-lineinfo"};
    const nvrtcResult rc = nvrtcCompileProgram(prog, 4, opts);
    if (rc != NVRTC_SUCCESS) {
        size_t logSize = 0;
        nvrtcGetProgramLogSize(prog, &logSize);
        std::string log(logSize, '\0');
        if (logSize) nvrtcGetProgramLog(prog, &log[0]);
        err = std::string(what) + " did not compile: " + nvrtcGetErrorString(rc) + "\n" + log;
        nvrtcDestroyProgram(&prog);
        return DEME_ERR_NVRTC;
    }
    size_t sz = 0;
    std::vector<char> cubin;
    std::string lowered;
    bool ok = nvrtcGetCUBINSize(prog, &sz) == NVRTC_SUCCESS && sz > 0;
    if (ok) {
        cubin.resize(sz);
        ok = nvrtcGetCUBIN(prog, cubin.data()) == NVRTC_SUCCESS;
    }
    const char* name = nullptr;
    ok = ok && nvrtcGetLoweredName(prog, expr, &name) == NVRTC_SUCCESS && name;
    if (ok) lowered = name;
    nvrtcDestroyProgram(&prog);
    if (!ok) {
        err = std::string("NVRTC produced no loadable image for the ") + what;
        return DEME_ERR_NVRTC;
    }
    lib = nullptr;
    kern = nullptr;
    if (cudaLibraryLoadData(&lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0) != cudaSuccess ||
        cudaLibraryGetKernel(&kern, lib, lowered.c_str()) != cudaSuccess) {
        err = std::string("loading the ") + what + " failed: " + cudaGetErrorString(cudaGetLastError());
        if (lib) cudaLibraryUnload(lib);
        lib = nullptr;
        kern = nullptr;
        return DEME_ERR_CUDA;
    }
    return DEME_OK;
}

}  // namespace

int32_t compile_family_change_rules(int32_t n, const uint32_t* from, const uint32_t* to,
                                    const char* const* conditions, FamilyChangeKernel& out, std::string& err) {
    if (n <= 0) {
        release_family_change_rules(out);
        return DEME_OK;
    }
    std::string inc;
    for (int32_t i = 0; i < n; i++) {
        if (!from || !to || !conditions || !conditions[i] || from[i] > 255u || to[i] > 255u) {
            err = "family change rule " + std::to_string(i) + ": families must lie in [0, 255] and the condition exist";
            return DEME_ERR_INVALID;
        }
        inc += "if (family_code == " + std::to_string(from[i]) + "u) {\nbool shouldMakeChange = false;\n{\n#line 1 \"" +
               "family_change_rule_" + std::to_string(i) + "\"\n" + returns_to_decision(conditions[i]) +
               "\n}\nif (shouldMakeChange) newFamily = " + std::to_string(to[i]) + "u;\n}\n";
    }
    FamilyChangeKernel k;
    const int32_t rc = build_one_kernel(kFamilySource, "deme_family_change.cu", {{"deme_family_change_rules.inc", inc}},
                                        "deme_b200::k_family_change", "family change rules", k.lib, k.kern, err);
    if (rc != DEME_OK) return rc;
    release_family_change_rules(out);
    out = k;
    return DEME_OK;
}

void release_family_change_rules(FamilyChangeKernel& k) {
    if (k.lib) cudaLibraryUnload(k.lib);
    k = FamilyChangeKernel{};
}

namespace {
const char* kMotionSource =
    "#include <stdint.h>\n"
    "#include \"force_model_api.cuh\"\n"
    "#include \"prescribed_motion_kernel.cuh\"\n";

// `<name> = <expression>;` under a #line naming the family and component, so the compiler log points at it.
void assign(std::string& out, int32_t family, const char* what, const char* name, const char* expr) {
    if (!expr) return;
    out += "\n#line 1 \"family_" + std::to_string(family) + "_" + what + "\"\n";
    out += std::string(name) + " = " + expr + ";\n";
}
}  // namespace

int32_t compile_prescribed_motion(int32_t n, const deme_motion_expressions* m, MotionKernel& out, std::string& err) {
    if (n <= 0) {
        release_prescribed_motion(out);
        return DEME_OK;
    }
    if (!m) {
        err = "prescribed motions: null array";
        return DEME_ERR_INVALID;
    }
    std::string vel, pos;
    std::vector<bool> seen(DEME_NUM_FAMILIES, false);
    for (int32_t i = 0; i < n; i++) {
        const deme_motion_expressions& e = m[i];
        if (e.family < 0 || e.family >= DEME_NUM_FAMILIES || seen[e.family]) {
            err = "prescribed motion " + std::to_string(i) + ": family must lie in [0, 255] and appear once";
            return DEME_ERR_INVALID;
        }
        seen[e.family] = true;
        static const char* kVel[3] = {"vX", "vY", "vZ"};
        static const char* kOmg[3] = {"omgBarX", "omgBarY", "omgBarZ"};
        static const char* kPos[3] = {"X", "Y", "Z"};
        static const char* kVelWhat[3] = {"lin_vel_x", "lin_vel_y", "lin_vel_z"};
        static const char* kOmgWhat[3] = {"ang_vel_x", "ang_vel_y", "ang_vel_z"};
        static const char* kPosWhat[3] = {"lin_pos_x", "lin_pos_y", "lin_pos_z"};
        const std::string head = "case " + std::to_string(e.family) + "u: {";
        vel += head;
        for (int c = 0; c < 3; c++) assign(vel, e.family, kVelWhat[c], kVel[c], e.lin_vel[c]);
        for (int c = 0; c < 3; c++) assign(vel, e.family, kOmgWhat[c], kOmg[c], e.ang_vel[c]);
        vel += "LinPrescribed = " + std::to_string(e.lin_vel_prescribed ? 1 : 0) + "; RotPrescribed = " +
               std::to_string(e.rot_vel_prescribed ? 1 : 0) + "; break; }\n";
        pos += head;
        for (int c = 0; c < 3; c++) assign(pos, e.family, kPosWhat[c], kPos[c], e.lin_pos[c]);
        pos += "LinPrescribed = " + std::to_string(e.lin_pos_prescribed ? 1 : 0) + "; RotPrescribed = " +
               std::to_string(e.rot_pos_prescribed ? 1 : 0) + "; break; }\n";
    }
    MotionKernel k;
    const int32_t rc = build_one_kernel(kMotionSource, "deme_prescribed_motion.cu",
                                        {{"deme_motion_vel.inc", vel}, {"deme_motion_pos.inc", pos}},
                                        "deme_b200::k_integrate_motion", "prescribed motion", k.lib, k.kern, err);
    if (rc != DEME_OK) return rc;
    release_prescribed_motion(out);
    out = k;
    return DEME_OK;
}

void release_prescribed_motion(MotionKernel& k) {
    if (k.lib) cudaLibraryUnload(k.lib);
    k = MotionKernel{};
}

}  // namespace deme_b200
