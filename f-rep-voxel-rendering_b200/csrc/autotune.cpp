// Batch autotuner and pool sizing, host C++ over the library's own C-ABI.
//
// The reference fixes one scene's branching by hand (gridDims,
// vulkan/src/main.cpp:16) and sizes its buffers for the worst case
// (voxel_storage.h:45-47: 512 MiB of tapes). A batch of hundreds of scenes
// needs both chosen per scene:
//   * frep_fit_pools voxelizes each scene once into a scratch tree per grid
//     (grown by doubling on overflow) and returns the node and tape words it
//     used plus a margin;
//   * frep_batch_autotune times batched voxelize + render (CUDA graph replay)
//     of a few scenes per class (effective resolution, tape-size class) under
//     each candidate branching and last-level tile, then the tapes (warps) per
//     block of the level passes on a mixed sample. Each candidate's figure is
//     the median of several timed runs, and a candidate replaces the
//     incumbent (the cached choice, else the default branching) only when it
//     is faster by a margin, so repeated tunings on the same device keep the
//     same choices.
// Tunings are saved as JSON keyed by device name (the format of the Python
// wrapper's cache, frep/autotune.py).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "capi_internal.h"

using frep::detail::cuda_fail;
using frep::detail::fail;

struct frep_tuning {
    struct Choice {
        std::vector<uint32_t> dims;
        uint32_t point_k = 0;
        float ms = NAN;
    };
    std::map<std::string, Choice> choices;  // "resolution:size class"
    uint32_t interval_warps = 0, point_warps = 0;
    bool warps_tuned = false;
};

namespace {

constexpr uint32_t kSizeClassBounds[3] = {256, 1024, 4096};

uint32_t size_class(uint32_t n_instr) {
    for (uint32_t i = 0; i < 3; i++)
        if (n_instr < kSizeClassBounds[i]) return i;
    return 3;
}

std::string class_key(uint32_t res, uint32_t n_instr) {
    return std::to_string(res) + ":" + std::to_string(size_class(n_instr));
}

// Candidate branchings per effective resolution: every level a multiple of 4
// from 4 to 32, two to four levels; the first is the default.
const std::vector<std::vector<uint32_t>>* candidates(uint32_t res) {
    static const std::map<uint32_t, std::vector<std::vector<uint32_t>>> table = {
        {64, {{16, 4}, {8, 8}, {4, 16}, {4, 4, 4}}},
        {128, {{16, 8}, {8, 16}, {32, 4}, {8, 4, 4}}},
        {256, {{16, 16}, {16, 4, 4}, {8, 8, 4}, {32, 8}}},
        {512, {{16, 8, 4}, {8, 8, 8}, {16, 32}, {32, 16}}},
        {1024, {{16, 16, 4}, {16, 8, 8}, {8, 8, 16}, {32, 8, 4}}},
    };
    auto it = table.find(res);
    return it == table.end() ? nullptr : &it->second;
}

frep_grid make_grid(const std::vector<uint32_t>& dims, const float* low, float world) {
    frep_grid g{};
    g.levels = (uint32_t)dims.size();
    for (size_t i = 0; i < dims.size(); i++) g.dims[i] = dims[i];
    for (int k = 0; k < 3; k++) g.low_vertex[k] = low[k];
    g.world_size = world;
    return g;
}

// Frees what one timing trial created, on every path.
struct Trial {
    std::vector<frep_tree*> trees;
    frep_batch* batch = nullptr;
    void* frames = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    ~Trial() {
        if (stream) cudaStreamSynchronize(stream);
        if (batch) frep_batch_destroy(batch);
        for (frep_tree* t : trees) frep_tree_destroy(t);
        if (frames) cudaFree(frames);
        for (cudaEvent_t e : ev)
            if (e) cudaEventDestroy(e);
        if (stream) cudaStreamDestroy(stream);
    }
};

struct Sample {
    std::vector<const frep_tape*> tapes;
    std::vector<frep_camera> cams;
    std::vector<frep_grid> grids;
    std::vector<uint32_t> ks;
};

// One timing of `s` with the given pools; `overflowed[i]` = tree i's
// overflow flags (1 nodes, 2 tapes) when the result is FREP_ERR_CAPACITY.
frep_status time_sample_with(frep_ctx* ctx, const Sample& s, const frep_lights* lights, uint32_t iw, uint32_t pw,
                             uint32_t reps, uint32_t W, uint32_t H, const std::vector<uint64_t>& nw,
                             const std::vector<uint64_t>& tw, std::vector<uint32_t>* overflowed, float* ms_out) {
    const uint32_t n = (uint32_t)s.tapes.size();
    frep_status st = FREP_OK;
    Trial tr;
    for (uint32_t i = 0; i < n; i++) {
        frep_voxelize_opts o{};
        o.rounding = FREP_ROUND_OUTWARD;
        o.shorten = 1;
        o.node_words = nw[i];
        o.tape_words = tw[i];
        o.point_cells_per_lane = s.ks[i];
        frep_tree* t = nullptr;
        st = frep_tree_create(ctx, &s.grids[i], &o, &t);
        if (st != FREP_OK) return st;
        tr.trees.push_back(t);
    }
    st = frep_batch_create(ctx, tr.trees.data(), n, &tr.batch);
    if (st != FREP_OK) return st;
    st = frep_batch_set_tuning(tr.batch, iw, pw);
    if (st != FREP_OK) return st;
    FREP_CUDA(cudaStreamCreateWithFlags(&tr.stream, cudaStreamNonBlocking));
    FREP_CUDA(cudaEventCreate(&tr.ev[0]));
    FREP_CUDA(cudaEventCreate(&tr.ev[1]));
    const size_t frame = (size_t)W * H * 4;
    if (cudaMalloc(&tr.frames, frame * n) != cudaSuccess) {
        tr.frames = nullptr;
        return fail(FREP_ERR_OOM, "frep_batch_autotune: frames of %u scenes", n);
    }
    std::vector<frep_image> imgs(n);
    std::vector<frep_camera> cams = s.cams;
    for (uint32_t i = 0; i < n; i++) {
        imgs[i].rgba8 = static_cast<uint8_t*>(tr.frames) + frame * i;
        imgs[i].hits = nullptr;
        cams[i].width = W;
        cams[i].height = H;
    }
    st = frep_batch_run(tr.batch, s.tapes.data(), nullptr, cams.data(), lights, imgs.data(), 1, tr.stream);
    if (st != FREP_OK) return st;
    std::vector<float> runs;
    for (uint32_t r = 0; r < reps; r++) {
        FREP_CUDA(cudaEventRecord(tr.ev[0], tr.stream));
        st = frep_batch_run(tr.batch, s.tapes.data(), nullptr, cams.data(), lights, imgs.data(), 1, tr.stream);
        if (st != FREP_OK) return st;
        FREP_CUDA(cudaEventRecord(tr.ev[1], tr.stream));
        FREP_CUDA(cudaEventSynchronize(tr.ev[1]));
        float ms = 0.0f;
        FREP_CUDA(cudaEventElapsedTime(&ms, tr.ev[0], tr.ev[1]));
        runs.push_back(ms);
    }
    overflowed->assign(n, 0u);
    frep_status worst = FREP_OK;
    for (uint32_t i = 0; i < n; i++) {
        frep_tree_info info{};
        st = frep_tree_sync(tr.trees[i], &info);
        if (st == FREP_ERR_CAPACITY) (*overflowed)[i] = info.overflow;
        else if (st != FREP_OK) return st;
        if (st != FREP_OK) worst = st;  // a pool that overflowed would time a partial tree
    }
    if (worst != FREP_OK) return worst;
    std::sort(runs.begin(), runs.end());
    *ms_out = runs[runs.size() / 2] / (float)n;
    return FREP_OK;
}

// Device ms per scene of batched voxelize + render of `s` (graph replay): the
// median of `reps` timed runs after one captured run. Pools are fitted from
// one voxelization of each scene alone plus `margin_pools`; a tree whose
// pool still overflows in the batched run gets that pool doubled and the
// sample is timed again (at most 4 times).
frep_status time_sample(frep_ctx* ctx, const Sample& s, const frep_lights* lights, uint32_t iw, uint32_t pw,
                        uint32_t reps, uint32_t W, uint32_t H, float margin_pools, float* ms_out) {
    const uint32_t n = (uint32_t)s.tapes.size();
    std::vector<uint64_t> nw(n), tw(n);
    frep_status st = frep_fit_pools(ctx, s.tapes.data(), s.grids.data(), nullptr, n, margin_pools, nw.data(),
                                    tw.data());
    if (st != FREP_OK) return st;
    std::vector<uint32_t> over;
    for (int attempt = 0;; attempt++) {
        st = time_sample_with(ctx, s, lights, iw, pw, reps, W, H, nw, tw, &over, ms_out);
        if (st != FREP_ERR_CAPACITY || attempt == 4) return st;
        for (uint32_t i = 0; i < n; i++) {
            if (over[i] & 1u) nw[i] *= 2;
            if (over[i] & 2u) tw[i] *= 2;
        }
    }
}

// ---- JSON of the tuning cache (the fixed schema frep/autotune.py writes) ----

struct Json {
    const std::string& s;
    size_t i = 0;
    explicit Json(const std::string& str) : s(str) {}
    void ws() {
        while (i < s.size() && (s[i] == ' ' || s[i] == '\n' || s[i] == '\t' || s[i] == '\r')) i++;
    }
    bool eat(char c) {
        ws();
        if (i < s.size() && s[i] == c) {
            i++;
            return true;
        }
        return false;
    }
    bool str(std::string* out) {
        ws();
        if (i >= s.size() || s[i] != '"') return false;
        i++;
        out->clear();
        while (i < s.size() && s[i] != '"') {
            if (s[i] == '\\' && i + 1 < s.size()) i++;
            out->push_back(s[i++]);
        }
        return i++ < s.size();
    }
    bool num(double* out) {
        ws();
        const char* b = s.c_str() + i;
        char* e = nullptr;
        if (s.compare(i, 3, "NaN") == 0) {
            *out = NAN;
            i += 3;
            return true;
        }
        *out = std::strtod(b, &e);
        if (e == b) return false;
        i += (size_t)(e - b);
        return true;
    }
    // Skips any value (for keys this reader does not use).
    bool skip() {
        ws();
        if (i >= s.size()) return false;
        if (s[i] == '"') {
            std::string t;
            return str(&t);
        }
        if (s[i] == '{' || s[i] == '[') {
            const char open = s[i], close = open == '{' ? '}' : ']';
            i++;
            if (eat(close)) return true;
            do {
                if (open == '{') {
                    std::string k;
                    if (!str(&k) || !eat(':')) return false;
                }
                if (!skip()) return false;
            } while (eat(','));
            return eat(close);
        }
        if (s.compare(i, 4, "true") == 0 || s.compare(i, 4, "null") == 0) {
            i += 4;
            return true;
        }
        if (s.compare(i, 5, "false") == 0) {
            i += 5;
            return true;
        }
        double d;
        return num(&d);
    }
};

bool parse_choice(Json& j, frep_tuning::Choice* c) {
    if (!j.eat('{')) return false;
    if (j.eat('}')) return true;
    do {
        std::string k;
        if (!j.str(&k) || !j.eat(':')) return false;
        if (k == "dims") {
            if (!j.eat('[')) return false;
            c->dims.clear();
            if (!j.eat(']')) {
                do {
                    double d;
                    if (!j.num(&d)) return false;
                    c->dims.push_back((uint32_t)d);
                } while (j.eat(','));
                if (!j.eat(']')) return false;
            }
        } else if (k == "point_cells_per_lane") {
            double d;
            if (!j.num(&d)) return false;
            c->point_k = (uint32_t)d;
        } else if (k == "ms_per_scene") {
            double d;
            if (!j.num(&d)) return false;
            c->ms = (float)d;
        } else if (!j.skip()) {
            return false;
        }
    } while (j.eat(','));
    return j.eat('}');
}

bool parse_entry(Json& j, frep_tuning* t) {
    if (!j.eat('{')) return false;
    if (j.eat('}')) return true;
    do {
        std::string k;
        if (!j.str(&k) || !j.eat(':')) return false;
        if (k == "choices") {
            if (!j.eat('{')) return false;
            if (!j.eat('}')) {
                do {
                    std::string key;
                    frep_tuning::Choice c;
                    if (!j.str(&key) || !j.eat(':') || !parse_choice(j, &c)) return false;
                    t->choices[key] = c;
                } while (j.eat(','));
                if (!j.eat('}')) return false;
            }
        } else if (k == "warps") {
            double a, b;
            if (!j.eat('[') || !j.num(&a) || !j.eat(',') || !j.num(&b) || !j.eat(']')) return false;
            t->interval_warps = (uint32_t)a;
            t->point_warps = (uint32_t)b;
            t->warps_tuned = true;
        } else if (!j.skip()) {
            return false;
        }
    } while (j.eat(','));
    return j.eat('}');
}

// The whole file as {device: raw entry text}, entries kept verbatim so that
// other devices' tunings survive a save.
bool split_devices(const std::string& text, std::map<std::string, std::string>* out) {
    Json j(text);
    if (!j.eat('{')) return false;
    if (j.eat('}')) return true;
    do {
        std::string dev;
        if (!j.str(&dev) || !j.eat(':')) return false;
        j.ws();
        const size_t b = j.i;
        if (!j.skip()) return false;
        (*out)[dev] = text.substr(b, j.i - b);
    } while (j.eat(','));
    return j.eat('}');
}

std::string json_string(const std::string& v) {
    std::string o = "\"";
    for (char c : v) {
        if (c == '"' || c == '\\') o.push_back('\\');
        o.push_back(c);
    }
    return o + "\"";
}

std::string entry_json(const frep_tuning* t) {
    std::ostringstream o;
    o << "{\n  \"choices\": {";
    bool first = true;
    for (const auto& kv : t->choices) {
        o << (first ? "\n" : ",\n") << "   " << json_string(kv.first) << ": {\"dims\": [";
        for (size_t i = 0; i < kv.second.dims.size(); i++) o << (i ? ", " : "") << kv.second.dims[i];
        o << "], \"point_cells_per_lane\": " << kv.second.point_k << ", \"ms_per_scene\": ";
        if (std::isnan(kv.second.ms)) o << "NaN";
        else o << kv.second.ms;
        o << "}";
        first = false;
    }
    o << (first ? "" : "\n  ") << "},\n  \"warps\": [" << t->interval_warps << ", " << t->point_warps << "]\n }";
    return o.str();
}

}  // namespace

extern "C" {

frep_status frep_fit_pools(frep_ctx* ctx, const frep_tape* const* tapes, const frep_grid* grids,
                           const float* tape_times, uint32_t n, float margin, uint64_t* node_words,
                           uint64_t* tape_words) {
    if (!ctx || (n && (!tapes || !grids || !node_words || !tape_words)))
        return fail(FREP_ERR_INVALID_ARG, "frep_fit_pools: null argument");
    if (!(margin >= 0.0f)) return fail(FREP_ERR_INVALID_ARG, "frep_fit_pools: margin %g", margin);
    std::map<std::vector<uint32_t>, std::pair<frep_tree*, uint64_t>> scratch;  // grid -> (tree, bytes)
    frep_status st = FREP_OK;
    for (uint32_t i = 0; i < n && st == FREP_OK; i++) {
        if (!tapes[i]) {
            st = fail(FREP_ERR_INVALID_ARG, "frep_fit_pools: tape %u is null", i);
            break;
        }
        std::vector<uint32_t> key(grids[i].dims, grids[i].dims + std::min<uint32_t>(grids[i].levels, FREP_MAX_LEVELS));
        key.push_back(grids[i].levels);
        for (;;) {
            auto& slot = scratch[key];
            if (!slot.first) {
                if (!slot.second) slot.second = 1ull << 30;
                frep_voxelize_opts o{};
                o.rounding = FREP_ROUND_OUTWARD;
                o.shorten = 1;
                o.node_words = slot.second / 4 / 4;
                o.tape_words = slot.second * 3 / 4 / 8;
                st = frep_tree_create(ctx, &grids[i], &o, &slot.first);
                if (st != FREP_OK) break;
            }
            st = frep_voxelize(ctx, slot.first, tapes[i], tape_times ? tape_times[i] : 0.0f, nullptr);
            if (st != FREP_OK) break;
            frep_tree_info info{};
            st = frep_tree_sync(slot.first, &info);
            if (st == FREP_OK) {
                node_words[i] = (uint64_t)((double)info.node_words_used * (1.0 + margin)) + 4096;
                tape_words[i] = (uint64_t)((double)info.tape_words_used * (1.0 + margin)) + 4096;
                break;
            }
            if (st != FREP_ERR_CAPACITY) break;
            frep_tree_destroy(slot.first);  // overflowed: twice the pools
            slot.first = nullptr;
            slot.second *= 2;
            if (slot.second > (1ull << 40)) {
                st = fail(FREP_ERR_CAPACITY, "frep_fit_pools: scene %u needs more than 1 TB of pools", i);
                break;
            }
            st = FREP_OK;
        }
    }
    for (auto& kv : scratch)
        if (kv.second.first) frep_tree_destroy(kv.second.first);
    return st;
}

frep_status frep_tuning_create(frep_tuning** out) {
    if (!out) return fail(FREP_ERR_INVALID_ARG, "frep_tuning_create: null argument");
    *out = new frep_tuning();
    return FREP_OK;
}

void frep_tuning_destroy(frep_tuning* t) { delete t; }

frep_status frep_tuning_load(frep_tuning* t, const char* path, const char* device) {
    if (!t || !path) return fail(FREP_ERR_INVALID_ARG, "frep_tuning_load: null argument");
    std::ifstream f(path, std::ios::binary);
    if (!f) return fail(FREP_ERR_INVALID_ARG, "frep_tuning_load: cannot open %s", path);
    std::stringstream ss;
    ss << f.rdbuf();
    std::map<std::string, std::string> devs;
    if (!split_devices(ss.str(), &devs)) return fail(FREP_ERR_INVALID_ARG, "frep_tuning_load: %s is not a tuning file", path);
    const std::string want = device ? device : "";
    auto it = devs.find(want);
    if (it == devs.end()) it = devs.find("NVIDIA B200");
    if (it == devs.end()) it = devs.begin();
    if (it == devs.end()) return FREP_OK;  // empty file: nothing tuned yet
    frep_tuning loaded;
    Json j(it->second);
    if (!parse_entry(j, &loaded)) return fail(FREP_ERR_INVALID_ARG, "frep_tuning_load: bad entry for %s", it->first.c_str());
    *t = loaded;
    return FREP_OK;
}

frep_status frep_tuning_save(const frep_tuning* t, const char* path, const char* device) {
    if (!t || !path || !device) return fail(FREP_ERR_INVALID_ARG, "frep_tuning_save: null argument");
    std::map<std::string, std::string> devs;
    {
        std::ifstream f(path, std::ios::binary);
        if (f) {
            std::stringstream ss;
            ss << f.rdbuf();
            if (!split_devices(ss.str(), &devs)) devs.clear();
        }
    }
    devs[device] = entry_json(t);
    std::ofstream o(path, std::ios::binary | std::ios::trunc);
    if (!o) return fail(FREP_ERR_INVALID_ARG, "frep_tuning_save: cannot write %s", path);
    o << "{";
    bool first = true;
    for (const auto& kv : devs) {
        o << (first ? "\n " : ",\n ") << json_string(kv.first) << ": " << kv.second;
        first = false;
    }
    o << "\n}\n";
    return o ? FREP_OK : fail(FREP_ERR_INVALID_ARG, "frep_tuning_save: write to %s failed", path);
}

frep_status frep_tuning_lookup(const frep_tuning* t, uint32_t resolution, uint32_t n_instr, uint32_t* levels,
                               uint32_t dims[FREP_MAX_LEVELS], uint32_t* point_cells_per_lane) {
    if (!t || !levels || !dims || !point_cells_per_lane)
        return fail(FREP_ERR_INVALID_ARG, "frep_tuning_lookup: null argument");
    auto it = t->choices.find(class_key(resolution, n_instr));
    if (it == t->choices.end() || it->second.dims.empty() || it->second.dims.size() > FREP_MAX_LEVELS) {
        *levels = 0;
        *point_cells_per_lane = 0;
        return FREP_OK;
    }
    *levels = (uint32_t)it->second.dims.size();
    for (uint32_t i = 0; i < FREP_MAX_LEVELS; i++) dims[i] = i < *levels ? it->second.dims[i] : 0;
    *point_cells_per_lane = it->second.point_k;
    return FREP_OK;
}

frep_status frep_tuning_warps(const frep_tuning* t, uint32_t* interval_warps_per_block,
                              uint32_t* point_warps_per_block) {
    if (!t || !interval_warps_per_block || !point_warps_per_block)
        return fail(FREP_ERR_INVALID_ARG, "frep_tuning_warps: null argument");
    *interval_warps_per_block = t->interval_warps;
    *point_warps_per_block = t->point_warps;
    return FREP_OK;
}

frep_status frep_batch_autotune(frep_ctx* ctx, const frep_tape* const* tapes, const uint32_t* resolutions,
                                const frep_camera* cameras, uint32_t n, const frep_lights* lights,
                                const float low_vertex[3], float world_size, const frep_autotune_opts* opts,
                                frep_tuning* tuning) {
    if (!ctx || !tuning || !lights || !low_vertex || (n && (!tapes || !resolutions || !cameras)))
        return fail(FREP_ERR_INVALID_ARG, "frep_batch_autotune: null argument");
    frep_autotune_opts o{};
    if (opts) o = *opts;
    const uint32_t per_class = o.per_class ? o.per_class : 4;
    const uint32_t reps = o.reps ? o.reps : 5;
    const uint32_t W = o.width ? o.width : 512, H = o.height ? o.height : 512;
    const float margin = o.margin > 0.0f ? o.margin : 0.03f;
    for (uint32_t i = 0; i < n; i++)
        if (!tapes[i] || !candidates(resolutions[i]))
            return fail(FREP_ERR_INVALID_ARG, "frep_batch_autotune: scene %u (resolution %u) has no candidate grid",
                        i, resolutions[i]);
    // classes in key order, members in input order
    std::map<std::string, std::vector<uint32_t>> classes;
    for (uint32_t i = 0; i < n; i++)
        classes[class_key(resolutions[i], (uint32_t)tapes[i]->ct.instrs.size())].push_back(i);
    for (const auto& kv : classes) {
        const bool cached = tuning->choices.count(kv.first) != 0;
        if (cached && !o.force && !o.refine) continue;
        const std::vector<uint32_t>& mem = kv.second;
        const uint32_t step = std::max<uint32_t>(1, (uint32_t)mem.size() / per_class);
        std::vector<uint32_t> pick;
        for (uint32_t i = 0; i < mem.size() && pick.size() < per_class; i += step) pick.push_back(mem[i]);
        const uint32_t res = resolutions[pick[0]];
        // the incumbent first: the cached choice, else the default branching
        std::vector<std::pair<std::vector<uint32_t>, uint32_t>> cands;
        if (cached && !o.force) cands.push_back({tuning->choices[kv.first].dims, tuning->choices[kv.first].point_k});
        for (const auto& d : *candidates(res)) {
            std::vector<uint32_t> ks = d.back() < 8 ? std::vector<uint32_t>{0} : std::vector<uint32_t>{4, 2};
            for (uint32_t k : ks)
                if (cands.empty() || !(cands[0].first == d && cands[0].second == k)) cands.push_back({d, k});
        }
        frep_tuning::Choice best;
        for (const auto& c : cands) {
            Sample s;
            for (uint32_t i : pick) {
                s.tapes.push_back(tapes[i]);
                s.cams.push_back(cameras[i]);
                s.grids.push_back(make_grid(c.first, low_vertex, world_size));
                s.ks.push_back(c.second);
            }
            float ms = 0.0f;
            frep_status st = time_sample(ctx, s, lights, tuning->interval_warps, tuning->point_warps, reps, W, H,
                                         0.02f, &ms);
            if (st != FREP_OK) return st;
            if (best.dims.empty() || ms < best.ms * (1.0f - margin)) best = frep_tuning::Choice{c.first, c.second, ms};
        }
        tuning->choices[kv.first] = best;
    }
    // tapes per block for the whole batch, on up to 32 scenes spread over it
    if (!tuning->warps_tuned || o.force || o.refine) {
        Sample s;
        const uint32_t step = std::max<uint32_t>(1, n / 32);
        for (uint32_t i = 0; i < n && s.tapes.size() < 32; i += step) {
            const auto& c = tuning->choices[class_key(resolutions[i], (uint32_t)tapes[i]->ct.instrs.size())];
            s.tapes.push_back(tapes[i]);
            s.cams.push_back(cameras[i]);
            s.grids.push_back(make_grid(c.dims, low_vertex, world_size));
            s.ks.push_back(c.point_k);
        }
        static const uint32_t kWarps[5][2] = {{0, 0}, {1, 1}, {4, 4}, {1, 4}, {4, 1}};
        std::vector<std::pair<uint32_t, uint32_t>> cands;
        if (tuning->warps_tuned && !o.force) cands.push_back({tuning->interval_warps, tuning->point_warps});
        for (const auto& w : kWarps)
            if (cands.empty() || !(cands[0].first == w[0] && cands[0].second == w[1])) cands.push_back({w[0], w[1]});
        float best_ms = 0.0f;
        std::pair<uint32_t, uint32_t> best{0, 0};
        bool have = false;
        for (const auto& w : cands) {
            float ms = 0.0f;
            if (!s.tapes.empty()) {
                frep_status st = time_sample(ctx, s, lights, w.first, w.second, reps, W, H, 0.02f, &ms);
                if (st != FREP_OK) return st;
            }
            if (!have || ms < best_ms * (1.0f - margin)) {
                best = w;
                best_ms = ms;
                have = true;
            }
        }
        tuning->interval_warps = best.first;
        tuning->point_warps = best.second;
        tuning->warps_tuned = true;
    }
    return FREP_OK;
}

}  // extern "C"
