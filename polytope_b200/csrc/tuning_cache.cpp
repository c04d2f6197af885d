// tuning_cache.cpp -- the batch autotuner's choices kept in a JSON file, keyed by the device and
// the class of the workload, so that a service tunes each kind of batch once per device instead of
// on every start (pt_tuning_class_of, pt_tuning_cache_get / _put, pt_batch_autotune_cached).
//
// File format (one object; entries in insertion order, a class appears at most once):
//   {"format": "polytope_b200 tuning cache", "version": 1,
//    "entries": [{"class": {"device": "...", "sm_count": 148, ...},
//                 "tuning": {"wave_pixels": ..., "threads_per_block": ..., ...}, "ms": 1.25}, ...]}
// Writers take an exclusive flock on "<path>.lock", read the file, replace or append their entry
// and rename a temporary file over the old one, so concurrent writers (threads or processes) keep
// each other's entries and readers always see a whole file.  A file that does not parse as this
// format is reported, never overwritten.

#include <fcntl.h>
#include <sys/file.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cerrno>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <set>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include <cuda_runtime.h>

#include "batch.h"
#include "pt_internal.h"

namespace pt {
namespace {

constexpr const char* kFormat = "polytope_b200 tuning cache";
constexpr double kVersion = 1;
constexpr size_t kMaxFileBytes = size_t(16) << 20;
constexpr int kMaxNesting = 16;

// ---- a small JSON reader (the subset RFC 8259 defines; depth-limited) ---------------------------
struct Json {
    enum Type { NUL, BOOL, NUM, STR, ARR, OBJ } type = NUL;
    bool b = false;
    double num = 0;
    std::string str;
    std::vector<Json> arr;
    std::vector<std::pair<std::string, Json>> obj;
    const Json* get(const char* key) const {
        for (const auto& kv : obj)
            if (kv.first == key) return &kv.second;
        return nullptr;
    }
};

class Reader {
public:
    Reader(const char* p, const char* end) : p_(p), end_(end) {}
    bool document(Json& out, std::string& why) {
        if (!value(out, 0)) { why = why_; return false; }
        ws();
        if (p_ != end_) { why = "trailing characters after the JSON value"; return false; }
        return true;
    }

private:
    const char *p_, *end_;
    std::string why_;
    bool err(const char* w) { if (why_.empty()) why_ = w; return false; }
    void ws() { while (p_ < end_ && (*p_ == ' ' || *p_ == '\t' || *p_ == '\n' || *p_ == '\r')) ++p_; }
    bool lit(const char* s) {
        const size_t n = std::strlen(s);
        if ((size_t)(end_ - p_) < n || std::memcmp(p_, s, n) != 0) return false;
        p_ += n;
        return true;
    }
    static void utf8(uint32_t c, std::string& o) {
        if (c < 0x80) o += (char)c;
        else if (c < 0x800) { o += (char)(0xC0 | (c >> 6)); o += (char)(0x80 | (c & 63)); }
        else if (c < 0x10000) { o += (char)(0xE0 | (c >> 12)); o += (char)(0x80 | ((c >> 6) & 63)); o += (char)(0x80 | (c & 63)); }
        else { o += (char)(0xF0 | (c >> 18)); o += (char)(0x80 | ((c >> 12) & 63)); o += (char)(0x80 | ((c >> 6) & 63)); o += (char)(0x80 | (c & 63)); }
    }
    bool hex4(uint32_t& v) {
        if (end_ - p_ < 4) return err("truncated \\u escape");
        v = 0;
        for (int k = 0; k < 4; ++k, ++p_) {
            const char c = *p_;
            v <<= 4;
            if (c >= '0' && c <= '9') v |= (uint32_t)(c - '0');
            else if (c >= 'a' && c <= 'f') v |= (uint32_t)(c - 'a' + 10);
            else if (c >= 'A' && c <= 'F') v |= (uint32_t)(c - 'A' + 10);
            else return err("bad \\u escape");
        }
        return true;
    }
    bool string(std::string& o) {
        ++p_;  // opening quote
        while (p_ < end_ && *p_ != '"') {
            const unsigned char c = (unsigned char)*p_;
            if (c < 0x20) return err("control character in a string");
            if (c != '\\') { o += (char)c; ++p_; continue; }
            if (++p_ >= end_) return err("truncated escape");
            const char e = *p_++;
            switch (e) {
                case '"': o += '"'; break;
                case '\\': o += '\\'; break;
                case '/': o += '/'; break;
                case 'b': o += '\b'; break;
                case 'f': o += '\f'; break;
                case 'n': o += '\n'; break;
                case 'r': o += '\r'; break;
                case 't': o += '\t'; break;
                case 'u': {
                    uint32_t c1;
                    if (!hex4(c1)) return false;
                    if (c1 >= 0xD800 && c1 < 0xDC00) {  // a surrogate pair
                        uint32_t c2;
                        if (!lit("\\u") || !hex4(c2) || c2 < 0xDC00 || c2 >= 0xE000) return err("unpaired surrogate");
                        c1 = 0x10000 + ((c1 - 0xD800) << 10) + (c2 - 0xDC00);
                    } else if (c1 >= 0xDC00 && c1 < 0xE000) {
                        return err("unpaired surrogate");
                    }
                    utf8(c1, o);
                    break;
                }
                default: return err("unknown escape");
            }
        }
        if (p_ >= end_) return err("unterminated string");
        ++p_;
        return true;
    }
    bool number(double& v) {
        const char* s = p_;
        if (p_ < end_ && *p_ == '-') ++p_;
        if (p_ >= end_ || !(*p_ >= '0' && *p_ <= '9')) return err("bad number");
        if (*p_ == '0') ++p_;
        else while (p_ < end_ && *p_ >= '0' && *p_ <= '9') ++p_;
        if (p_ < end_ && *p_ == '.') {
            ++p_;
            if (p_ >= end_ || !(*p_ >= '0' && *p_ <= '9')) return err("bad number");
            while (p_ < end_ && *p_ >= '0' && *p_ <= '9') ++p_;
        }
        if (p_ < end_ && (*p_ == 'e' || *p_ == 'E')) {
            ++p_;
            if (p_ < end_ && (*p_ == '+' || *p_ == '-')) ++p_;
            if (p_ >= end_ || !(*p_ >= '0' && *p_ <= '9')) return err("bad number");
            while (p_ < end_ && *p_ >= '0' && *p_ <= '9') ++p_;
        }
        // from_chars, unlike strtod, ignores the process locale (a decimal comma would cut "1.5")
        const std::from_chars_result r = std::from_chars(s, p_, v);
        if (r.ec == std::errc::result_out_of_range) return err("number out of range");
        if (r.ec != std::errc() || r.ptr != p_) return err("bad number");
        return true;
    }
    bool value(Json& v, int depth) {
        if (depth > kMaxNesting) return err("nesting too deep");
        ws();
        if (p_ >= end_) return err("unexpected end of file");
        const char c = *p_;
        if (c == '{') {
            v.type = Json::OBJ;
            ++p_;
            ws();
            if (p_ < end_ && *p_ == '}') { ++p_; return true; }
            for (;;) {
                ws();
                if (p_ >= end_ || *p_ != '"') return err("expected a key");
                std::string key;
                if (!string(key)) return false;
                ws();
                if (p_ >= end_ || *p_ != ':') return err("expected ':'");
                ++p_;
                Json item;
                if (!value(item, depth + 1)) return false;
                v.obj.emplace_back(std::move(key), std::move(item));
                ws();
                if (p_ < end_ && *p_ == ',') { ++p_; continue; }
                if (p_ < end_ && *p_ == '}') { ++p_; return true; }
                return err("expected ',' or '}'");
            }
        }
        if (c == '[') {
            v.type = Json::ARR;
            ++p_;
            ws();
            if (p_ < end_ && *p_ == ']') { ++p_; return true; }
            for (;;) {
                Json item;
                if (!value(item, depth + 1)) return false;
                v.arr.push_back(std::move(item));
                ws();
                if (p_ < end_ && *p_ == ',') { ++p_; continue; }
                if (p_ < end_ && *p_ == ']') { ++p_; return true; }
                return err("expected ',' or ']'");
            }
        }
        if (c == '"') { v.type = Json::STR; return string(v.str); }
        if (lit("true")) { v.type = Json::BOOL; v.b = true; return true; }
        if (lit("false")) { v.type = Json::BOOL; v.b = false; return true; }
        if (lit("null")) { v.type = Json::NUL; return true; }
        v.type = Json::NUM;
        return number(v.num);
    }
};

// ---- entries --------------------------------------------------------------------------------------
struct Entry {
    pt_tuning_class cls;
    pt_batch_tuning tuning;
    double ms;
};

// The class's integer fields, in file order.
struct UField { const char* name; uint32_t pt_tuning_class::*member; };
const UField kClassFields[] = {
    {"sm_count", &pt_tuning_class::sm_count},         {"compute_capability", &pt_tuning_class::compute_capability},
    {"items_log2", &pt_tuning_class::items_log2},     {"pixels_log2", &pt_tuning_class::pixels_log2},
    {"samples_log2", &pt_tuning_class::samples_log2}, {"faces_log2", &pt_tuning_class::faces_log2},
    {"tree_depth", &pt_tuning_class::tree_depth},     {"max_depth", &pt_tuning_class::max_depth},
    {"flags", &pt_tuning_class::flags},
};
struct TField { const char* name; uint32_t pt_batch_tuning::*member; };
const TField kTuningFields[] = {
    {"threads_per_block", &pt_batch_tuning::threads_per_block}, {"stack_depth", &pt_batch_tuning::stack_depth},
    {"queue_chunk", &pt_batch_tuning::queue_chunk},             {"pipeline", &pt_batch_tuning::pipeline},
};

size_t device_len(const pt_tuning_class& c) {  // length of the NUL-terminated name; 64 if unterminated
    const void* nul = std::memchr(c.device, 0, sizeof(c.device));
    return nul ? (size_t)(static_cast<const char*>(nul) - c.device) : sizeof(c.device);
}

bool same_class(const pt_tuning_class& a, const pt_tuning_class& b) {
    if (std::strncmp(a.device, b.device, sizeof(a.device)) != 0) return false;
    for (const auto& f : kClassFields)
        if (a.*(f.member) != b.*(f.member)) return false;
    return true;
}

int check_class(const pt_tuning_class& c) {
    const size_t n = device_len(c);
    if (n == 0 || n >= sizeof(c.device)) return fail(PT_EINVAL, "tuning class: device name empty or not NUL-terminated");
    return PT_OK;
}

bool as_uint(const Json* v, double limit, double& out) {
    if (!v || v->type != Json::NUM || !(v->num >= 0) || v->num > limit || std::floor(v->num) != v->num) return false;
    out = v->num;
    return true;
}

int entry_from_json(const Json& e, size_t index, Entry& out, const std::string& path) {
    const std::string at = path + ": entry " + std::to_string(index) + ": ";
    if (e.type != Json::OBJ) return fail(PT_EINVAL, at + "not an object");
    const Json* c = e.get("class");
    const Json* t = e.get("tuning");
    const Json* ms = e.get("ms");
    if (!c || c->type != Json::OBJ || !t || t->type != Json::OBJ) return fail(PT_EINVAL, at + "needs \"class\" and \"tuning\" objects");
    if (!ms || ms->type != Json::NUM || !std::isfinite(ms->num) || ms->num < 0) return fail(PT_EINVAL, at + "\"ms\" must be a number >= 0");
    out = Entry{};
    const Json* dev = c->get("device");
    if (!dev || dev->type != Json::STR || dev->str.empty() || dev->str.size() >= sizeof(out.cls.device) ||
        dev->str.find('\0') != std::string::npos)
        return fail(PT_EINVAL, at + "class.device must be a string of 1-63 bytes");
    std::memcpy(out.cls.device, dev->str.data(), dev->str.size());
    double v = 0;
    for (const auto& f : kClassFields) {
        if (!as_uint(c->get(f.name), 4294967295.0, v)) return fail(PT_EINVAL, at + "class." + f.name + " must be an integer in [0, 2^32)");
        out.cls.*(f.member) = (uint32_t)v;
    }
    if (!as_uint(t->get("wave_pixels"), 9007199254740992.0, v)) return fail(PT_EINVAL, at + "tuning.wave_pixels must be an integer in [0, 2^53]");
    out.tuning.wave_pixels = (uint64_t)v;
    for (const auto& f : kTuningFields) {
        if (!as_uint(t->get(f.name), 4294967295.0, v)) return fail(PT_EINVAL, at + "tuning." + f.name + " must be an integer in [0, 2^32)");
        out.tuning.*(f.member) = (uint32_t)v;
    }
    if (check_tuning(out.tuning) != PT_OK) return fail(PT_EINVAL, at + pt_last_error());
    out.ms = ms->num;
    return PT_OK;
}

void put_string(std::string& o, const char* s, size_t n) {
    o += '"';
    for (size_t i = 0; i < n; ++i) {
        const unsigned char c = (unsigned char)s[i];
        if (c == '"' || c == '\\') { o += '\\'; o += (char)c; }
        else if (c < 0x20) { char b[8]; std::snprintf(b, sizeof(b), "\\u%04x", c); o += b; }
        else o += (char)c;
    }
    o += '"';
}

std::string to_json(const std::vector<Entry>& entries) {
    std::string o = "{\"format\": ";
    put_string(o, kFormat, std::strlen(kFormat));
    o += ", \"version\": 1, \"entries\": [";
    char b[64];
    for (size_t i = 0; i < entries.size(); ++i) {
        const Entry& e = entries[i];
        o += i ? ",\n  " : "\n  ";
        o += "{\"class\": {\"device\": ";
        put_string(o, e.cls.device, device_len(e.cls));
        for (const auto& f : kClassFields) {
            std::snprintf(b, sizeof(b), ", \"%s\": %u", f.name, (unsigned)(e.cls.*(f.member)));
            o += b;
        }
        std::snprintf(b, sizeof(b), "}, \"tuning\": {\"wave_pixels\": %llu", (unsigned long long)e.tuning.wave_pixels);
        o += b;
        for (const auto& f : kTuningFields) {
            std::snprintf(b, sizeof(b), ", \"%s\": %u", f.name, (unsigned)(e.tuning.*(f.member)));
            o += b;
        }
        // the shortest text that reads back to the same double, whatever the process locale
        o += "}, \"ms\": ";
        const std::to_chars_result r = std::to_chars(b, b + sizeof(b), e.ms);
        o.append(b, r.ptr);
        o += '}';
    }
    o += entries.empty() ? "]}\n" : "\n]}\n";
    return o;
}

// Reads the cache at `path` into `out`.  A missing file is an empty cache; anything that is not
// this format is PT_EINVAL with the reason.
int load(const std::string& path, std::vector<Entry>& out) {
    out.clear();
    const int fd = ::open(path.c_str(), O_RDONLY | O_CLOEXEC);
    if (fd < 0) {
        if (errno == ENOENT) return PT_OK;
        return fail(PT_EINVAL, path + ": " + std::strerror(errno));
    }
    struct stat st;
    if (::fstat(fd, &st) != 0 || !S_ISREG(st.st_mode) || (size_t)st.st_size > kMaxFileBytes) {
        ::close(fd);
        return fail(PT_EINVAL, path + ": not a regular file of at most 16 MiB");
    }
    std::string text((size_t)st.st_size, '\0');
    size_t got = 0;
    while (got < text.size()) {
        const ssize_t r = ::read(fd, &text[got], text.size() - got);
        if (r < 0 && errno == EINTR) continue;
        if (r <= 0) break;
        got += (size_t)r;
    }
    ::close(fd);
    text.resize(got);
    Json doc;
    std::string why;
    if (!Reader(text.data(), text.data() + text.size()).document(doc, why)) return fail(PT_EINVAL, path + ": " + why);
    const Json* fmt = doc.get("format");
    const Json* ver = doc.get("version");
    const Json* ents = doc.get("entries");
    if (doc.type != Json::OBJ || !fmt || fmt->type != Json::STR || fmt->str != kFormat)
        return fail(PT_EINVAL, path + ": not a polytope_b200 tuning cache");
    if (!ver || ver->type != Json::NUM || ver->num != kVersion) return fail(PT_EINVAL, path + ": unsupported version");
    if (!ents || ents->type != Json::ARR) return fail(PT_EINVAL, path + ": \"entries\" must be an array");
    out.resize(ents->arr.size());
    for (size_t i = 0; i < ents->arr.size(); ++i) {
        const int rc = entry_from_json(ents->arr[i], i, out[i], path);
        if (rc) return rc;
    }
    return PT_OK;
}

struct FileLock {  // exclusive advisory lock on "<path>.lock" for the read-modify-write of a put
    int fd = -1;
    ~FileLock() {
        if (fd >= 0) { ::flock(fd, LOCK_UN); ::close(fd); }
    }
    int take(const std::string& path) {
        fd = ::open((path + ".lock").c_str(), O_RDWR | O_CREAT | O_CLOEXEC, 0644);
        if (fd < 0) return fail(PT_EINVAL, path + ".lock: " + std::strerror(errno));
        while (::flock(fd, LOCK_EX) != 0) {
            if (errno != EINTR) return fail(PT_EINVAL, path + ".lock: " + std::strerror(errno));
        }
        return PT_OK;
    }
};

int store(const std::string& path, const std::vector<Entry>& entries) {
    const std::string text = to_json(entries);
    char suffix[64];
    std::snprintf(suffix, sizeof(suffix), ".tmp.%d.%zx", (int)::getpid(), std::hash<std::thread::id>()(std::this_thread::get_id()));
    const std::string tmp = path + suffix;
    const int fd = ::open(tmp.c_str(), O_WRONLY | O_CREAT | O_TRUNC | O_CLOEXEC, 0644);
    if (fd < 0) return fail(PT_EINVAL, tmp + ": " + std::strerror(errno));
    size_t put = 0;
    while (put < text.size()) {
        const ssize_t w = ::write(fd, text.data() + put, text.size() - put);
        if (w < 0 && errno == EINTR) continue;
        if (w <= 0) break;
        put += (size_t)w;
    }
    const bool ok = put == text.size() && ::fsync(fd) == 0;
    ::close(fd);
    if (!ok || ::rename(tmp.c_str(), path.c_str()) != 0) {
        const std::string why = std::strerror(errno);
        ::unlink(tmp.c_str());
        return fail(PT_EINVAL, path + ": write failed: " + why);
    }
    return PT_OK;
}

uint32_t floor_log2(uint64_t v) {
    uint32_t r = 0;
    while (v >>= 1) ++r;
    return r;
}

}  // namespace
}  // namespace pt

using namespace pt;

extern "C" int pt_tuning_class_of(const pt_batch_item* items, uint32_t n, pt_tuning_class* cls) {
    if (!items || !n || !cls) return fail(PT_EINVAL, "items or cls is NULL");
    pt_tuning_class c{};
    uint64_t pixels = 0, samples = 0, faces = 0;
    std::set<const pt_scene*> seen;
    for (uint32_t i = 0; i < n; ++i) {
        const pt_scene* s = items[i].scene;
        if (!s) return fail(PT_EINVAL, "item " + std::to_string(i) + ": NULL scene");
        const pt_render_desc& d = items[i].desc;
        pixels += (uint64_t)d.width * d.height;
        samples += (uint64_t)d.width * d.height * d.spp;
        c.tree_depth = std::max(c.tree_depth, s->max_depth);
        c.max_depth = std::max(c.max_depth, d.max_depth);
        c.flags |= d.flags;
        if (seen.insert(s).second) faces += s->num_prims;
    }
    c.items_log2 = floor_log2(n);
    c.pixels_log2 = floor_log2(pixels);
    c.samples_log2 = floor_log2(samples);
    c.faces_log2 = floor_log2(faces);
    cudaDeviceProp p;
    const cudaError_t e = cudaGetDeviceProperties(&p, items[0].scene->device);
    if (e != cudaSuccess) return fail(PT_ECUDA, std::string("cudaGetDeviceProperties: ") + cudaGetErrorString(e));
    const size_t name_len = std::min(strnlen(p.name, sizeof(p.name)), sizeof(c.device) - 1);
    std::memcpy(c.device, p.name, name_len);  // c.device is zeroed, so the name stays terminated
    c.sm_count = (uint32_t)p.multiProcessorCount;
    c.compute_capability = (uint32_t)(p.major * 10 + p.minor);
    *cls = c;
    return PT_OK;
}

extern "C" int pt_tuning_cache_get(const char* path, const pt_tuning_class* cls, pt_batch_tuning* tuning, double* ms,
                                   int* found) {
    if (!path || !cls || !tuning || !found) return fail(PT_EINVAL, "path, cls, tuning or found is NULL");
    *found = 0;
    int rc = check_class(*cls);
    if (rc) return rc;
    std::vector<Entry> entries;
    rc = load(path, entries);
    if (rc) return rc;
    for (const Entry& e : entries) {
        if (!same_class(e.cls, *cls)) continue;
        *tuning = e.tuning;
        if (ms) *ms = e.ms;
        *found = 1;
        break;
    }
    return PT_OK;
}

extern "C" int pt_tuning_cache_put(const char* path, const pt_tuning_class* cls, const pt_batch_tuning* tuning,
                                   double ms) {
    if (!path || !*path || !cls || !tuning) return fail(PT_EINVAL, "path, cls or tuning is NULL");
    int rc = check_class(*cls);
    if (rc) return rc;
    if (check_tuning(*tuning) != PT_OK) return PT_EINVAL;
    if (!std::isfinite(ms) || ms < 0) return fail(PT_EINVAL, "ms must be a finite number >= 0");
    FileLock lock;
    rc = lock.take(path);
    if (rc) return rc;
    std::vector<Entry> entries;
    rc = load(path, entries);  // a file that is not a tuning cache is reported, not replaced
    if (rc) return rc;
    Entry mine{};
    mine.cls = *cls;
    std::memset(mine.cls.device, 0, sizeof(mine.cls.device));
    std::memcpy(mine.cls.device, cls->device, device_len(*cls));
    mine.tuning = *tuning;
    mine.ms = ms;
    bool placed = false;
    std::vector<Entry> kept;
    kept.reserve(entries.size() + 1);
    for (const Entry& e : entries) {
        if (!same_class(e.cls, mine.cls)) { kept.push_back(e); continue; }
        if (!placed) { kept.push_back(mine); placed = true; }
    }
    if (!placed) kept.push_back(mine);
    return store(path, kept);
}

extern "C" int pt_batch_autotune_cached(const pt_batch_item* items, uint32_t n, const char* path, pt_batch_tuning* best,
                                        double* best_ms, int* from_cache) {
    if (!items || !n || !path || !best) return fail(PT_EINVAL, "items, path or best is NULL");
    if (from_cache) *from_cache = 0;
    pt_tuning_class cls;
    int rc = pt_tuning_class_of(items, n, &cls);
    if (rc) return rc;
    pt_batch_tuning t;
    double ms = 0;
    int found = 0;
    rc = pt_tuning_cache_get(path, &cls, &t, &ms, &found);
    if (rc) return rc;
    if (!found) {
        rc = pt_batch_autotune(items, n, &t, &ms, nullptr, nullptr);
        if (rc) return rc;
    }
    *best = t;
    if (best_ms) *best_ms = ms;
    if (found) {
        if (from_cache) *from_cache = 1;
        return PT_OK;
    }
    return pt_tuning_cache_put(path, &cls, &t, ms);
}
