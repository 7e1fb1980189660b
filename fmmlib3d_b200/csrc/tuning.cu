// The autotuner's JSON cache (reader) and the device tag of the signatures.
//
// Cache format, written by fmmlib3d_b200/autotune.py:
//   {"format": "fmm3d_b200 tuning cache", "version": 1,
//    "entries": {"<signature>": {"knobs": {"m2l_kt": 64, "trans_kt": 8, "tc_variant": 1,
//                                          "overlap": 1, "p2p_ept": 4}, "ms": ..., ...}, ...}}
// Only "entries" / <signature> / "knobs" is read; other fields are for people.
#include <dlfcn.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/fmm3d_b200.h"
#include "tuning.cuh"

namespace fmm {

namespace {

// ------------------------------------------------------------ minimal JSON reader
struct JVal {
    enum Kind { Null, Bool, Num, Str, Arr, Obj } kind = Null;
    double num = 0;
    std::string str;
    std::vector<JVal> arr;
    std::vector<std::pair<std::string, JVal>> obj;
    const JVal *get(const char *key) const
    {
        if (kind != Obj) return nullptr;
        for (auto &kv : obj)
            if (kv.first == key) return &kv.second;
        return nullptr;
    }
};

struct JParser {
    const std::string &s;
    size_t i = 0;
    bool ok = true;
    explicit JParser(const std::string &text) : s(text) {}
    void ws()
    {
        while (i < s.size() && (s[i] == ' ' || s[i] == '\t' || s[i] == '\n' || s[i] == '\r')) i++;
    }
    bool lit(const char *w)
    {
        size_t n = strlen(w);
        if (s.compare(i, n, w) != 0) return false;
        i += n;
        return true;
    }
    std::string string()
    {
        std::string out;
        if (i >= s.size() || s[i] != '"') { ok = false; return out; }
        i++;
        while (i < s.size() && s[i] != '"') {
            char c = s[i++];
            if (c == '\\' && i < s.size()) {
                char e = s[i++];
                switch (e) {
                case 'n': out += '\n'; break;
                case 't': out += '\t'; break;
                case 'r': out += '\r'; break;
                case 'b': out += '\b'; break;
                case 'f': out += '\f'; break;
                case 'u':   // non-ASCII code points are not used in signatures
                    if (i + 4 <= s.size()) {
                        unsigned v = (unsigned)strtoul(s.substr(i, 4).c_str(), nullptr, 16);
                        out += v < 128 ? (char)v : '?';
                        i += 4;
                    } else {
                        ok = false;
                    }
                    break;
                default: out += e;
                }
            } else {
                out += c;
            }
        }
        if (i >= s.size()) { ok = false; return out; }
        i++;
        return out;
    }
    JVal value(int depth)
    {
        JVal v;
        ws();
        if (!ok || i >= s.size() || depth > 64) { ok = false; return v; }
        char c = s[i];
        if (c == '{') {
            v.kind = JVal::Obj;
            i++;
            ws();
            if (i < s.size() && s[i] == '}') { i++; return v; }
            while (ok) {
                ws();
                std::string k = string();
                ws();
                if (!ok || i >= s.size() || s[i] != ':') { ok = false; break; }
                i++;
                JVal x = value(depth + 1);
                v.obj.emplace_back(std::move(k), std::move(x));
                ws();
                if (i < s.size() && s[i] == ',') { i++; continue; }
                if (i < s.size() && s[i] == '}') { i++; break; }
                ok = false;
            }
        } else if (c == '[') {
            v.kind = JVal::Arr;
            i++;
            ws();
            if (i < s.size() && s[i] == ']') { i++; return v; }
            while (ok) {
                v.arr.push_back(value(depth + 1));
                ws();
                if (i < s.size() && s[i] == ',') { i++; continue; }
                if (i < s.size() && s[i] == ']') { i++; break; }
                ok = false;
            }
        } else if (c == '"') {
            v.kind = JVal::Str;
            v.str = string();
        } else if (lit("true")) {
            v.kind = JVal::Bool; v.num = 1;
        } else if (lit("false")) {
            v.kind = JVal::Bool;
        } else if (lit("null")) {
            v.kind = JVal::Null;
        } else {
            const char *b = s.c_str() + i;
            char *e = nullptr;
            v.num = strtod(b, &e);
            if (e == b) { ok = false; return v; }
            v.kind = JVal::Num;
            i += (size_t)(e - b);
        }
        return v;
    }
};

// ------------------------------------------------------------ the cache
std::mutex g_tune_mu;
bool g_path_set = false;          // fmm3d_set_tuning_cache was called
std::string g_path_override;
bool g_loaded = false;
std::string g_loaded_path;
std::map<std::string, TuneKnobs> g_entries;

std::string library_dir()
{
    Dl_info info;
    if (dladdr((void *)&library_dir, &info) && info.dli_fname) {
        std::string f = info.dli_fname;
        size_t k = f.find_last_of('/');
        return k == std::string::npos ? std::string(".") : f.substr(0, k);
    }
    return ".";
}

std::string cache_path()
{
    if (g_path_set) return g_path_override;
    if (const char *e = getenv("FMM3D_TUNING_CACHE")) return e;
    return library_dir() + "/tuning_cache.json";
}

void load_locked()
{
    const std::string path = cache_path();
    if (g_loaded && path == g_loaded_path) return;
    g_entries.clear();
    g_loaded = true;
    g_loaded_path = path;
    if (path.empty() || path == "none") return;
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) return;
    std::string text;
    char buf[65536];
    size_t n;
    while ((n = fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, n);
    fclose(f);
    JParser P(text);
    JVal root = P.value(0);
    P.ws();
    if (!P.ok || P.i != text.size()) return;   // an unreadable cache is ignored (automatic knobs)
    const JVal *ents = root.get("entries");
    if (!ents || ents->kind != JVal::Obj) return;
    static const char *names[kNumKnobs] = {"m2l_kt", "trans_kt", "tc_variant", "overlap", "p2p_ept"};
    for (auto &kv : ents->obj) {
        const JVal *kn = kv.second.get("knobs");
        if (!kn || kn->kind != JVal::Obj) continue;
        int a[kNumKnobs] = {0, 0, 0, 0, 0};
        for (int j = 0; j < kNumKnobs; j++) {
            const JVal *x = kn->get(names[j]);
            if (x && x->kind == JVal::Num && x->num >= 0 && x->num <= 1024) a[j] = (int)x->num;
        }
        g_entries[kv.first] = knobs_from_array(a);
    }
}

}  // namespace

bool tuning_lookup(const std::string &signature, TuneKnobs &k)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    load_locked();
    auto it = g_entries.find(signature);
    if (it == g_entries.end()) return false;
    k = it->second;
    return true;
}

std::string device_tag()
{
    // cudaGetDeviceProperties takes milliseconds: once per device
    static std::mutex mu;
    static std::map<int, std::string> tags;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(mu);
    auto it = tags.find(dev);
    if (it != tags.end()) return it->second;
    int sms = 0;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return "unknown";
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return tags[dev] = std::string(prop.name) + "/" + std::to_string(sms);
}

int log2_bucket(long long n)
{
    return n <= 0 ? 0 : (int)lround(log2((double)n));
}

}  // namespace fmm

using namespace fmm;

extern "C" {

int fmm3d_set_tuning_cache(const char *path)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_path_set = path != nullptr;
    g_path_override = path ? path : "";
    g_loaded = false;
    return 0;
}

int fmm3d_tuning_reload(void)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_loaded = false;
    load_locked();
    return (int)g_entries.size();
}

int fmm3d_tuning_cache_path(char *buf, int n)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    std::string p = cache_path();
    if (!buf || n <= 0) return (int)p.size() + 1;
    snprintf(buf, (size_t)n, "%s", p.c_str());
    return (int)p.size() + 1 <= n ? 0 : (int)p.size() + 1;
}

}  // extern "C"
