// `.inp` preprocessing and keyword parser with the semantics of FerriX's
// src/solver/parser.rs (keyword state machine :111-482, data lines :484-876,
// argument helpers :879-894, preprocessing :903-942), node / element line
// parsing (mesh_lib/node.rs:25-35, mesh_lib/elements/element.rs:62-131) and
// the node mapping of mesh_lib/mesh.rs:35-50.
//
// Reproduced behaviour: only the first data line after *BOUNDARY and
// *AMPLITUDE is read; data following an ignored keyword is dropped; DOFs 4-6
// are dropped; a *CLOAD on an nset gives the full value to every node; loads
// and BCs carry over between steps unless OP=NEW; unknown keywords are an
// error. Case folding is ASCII (decks are ASCII).
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <deque>
#include <functional>
#include <memory>
#include <mutex>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <unordered_set>

#include <charconv>
#include <string_view>
#include <thread>

#include <unistd.h>

#include "common.hpp"
#include "model.hpp"

namespace fx {

// ------------------------------------------------------------------ helpers

static inline bool is_ws(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\n' || c == '\v' || c == '\f'; }

static std::string trim(const std::string& s) {
    size_t a = 0, b = s.size();
    while (a < b && is_ws(s[a])) ++a;
    while (b > a && is_ws(s[b - 1])) --b;
    return s.substr(a, b - a);
}

static std::vector<std::string> split(const std::string& s, char sep) {
    std::vector<std::string> out;
    size_t start = 0;
    for (size_t i = 0; i <= s.size(); ++i) {
        if (i == s.size() || s[i] == sep) {
            out.push_back(s.substr(start, i - start));
            start = i + 1;
        }
    }
    return out;
}

static bool starts_with(const std::string& s, const char* p) { return s.rfind(p, 0) == 0; }

// f64::from_str: decimal / exponent forms, inf / infinity / nan; nothing else.
static bool parse_f64_slow(const std::string& s, double* out) {
    if (s.empty()) return false;
    std::string low;
    for (char c : s) low.push_back((char)std::tolower((unsigned char)c));
    size_t i = (low[0] == '+' || low[0] == '-') ? 1 : 0;
    std::string body = low.substr(i);
    if (body == "inf" || body == "infinity" || body == "nan") {
        double v = body == "nan" ? NAN : INFINITY;
        *out = low[0] == '-' ? -v : v;
        return true;
    }
    bool digit = false;
    for (size_t k = i; k < low.size(); ++k) {
        char c = low[k];
        if (std::isdigit((unsigned char)c)) digit = true;
        else if (!(c == '.' || c == 'e' || c == '+' || c == '-')) return false;
    }
    if (!digit) return false;
    char* end = nullptr;
    errno = 0;
    double v = std::strtod(s.c_str(), &end);
    if (end != s.c_str() + s.size()) return false;
    *out = v;
    return true;
}

// usize::from_str: optional '+', ASCII digits, no overflow.
static bool parse_usize(const std::string& s, int64_t* out) {
    size_t i = 0;
    if (!s.empty() && s[0] == '+') i = 1;
    if (i >= s.size()) return false;
    uint64_t v = 0;
    for (; i < s.size(); ++i) {
        if (!std::isdigit((unsigned char)s[i])) return false;
        uint64_t d = (uint64_t)(s[i] - '0');
        if (v > (UINT64_MAX - d) / 10) return false;
        v = v * 10 + d;
    }
    if (v > (uint64_t)INT64_MAX) return false;
    *out = (int64_t)v;
    return true;
}

// Allocation-free forms for the bulk data lines (*NODE, *ELEMENT): fields as
// views into the line, trimmed like trim().
static void split_views(std::string_view s, char sep, std::vector<std::string_view>& out) {
    out.clear();
    size_t start = 0;
    for (size_t i = 0; i <= s.size(); ++i) {
        if (i == s.size() || s[i] == sep) {
            size_t a = start, b = i;
            while (a < b && is_ws(s[a])) ++a;
            while (b > a && is_ws(s[b - 1])) --b;
            out.emplace_back(s.data() + a, b - a);
            start = i + 1;
        }
    }
}

static bool parse_usize_sv(std::string_view s, int64_t* out) {  // usize::from_str
    size_t i = 0;
    if (!s.empty() && s[0] == '+') i = 1;
    if (i >= s.size()) return false;
    uint64_t v = 0;
    for (; i < s.size(); ++i) {
        const unsigned d = (unsigned)(s[i] - '0');
        if (d > 9) return false;
        if (v > (UINT64_MAX - d) / 10) return false;
        v = v * 10 + d;
    }
    if (v > (uint64_t)INT64_MAX) return false;
    *out = (int64_t)v;
    return true;
}

// f64::from_str without allocation: same accepted forms as parse_f64 below.
static bool parse_f64_sv(std::string_view s, double* out) {
    // the usual decimal forms: a complete, finite from_chars parse (no leading '+', which
    // from_chars does not take; inf / nan spellings and out-of-range values are not finite
    // or fail, and go through the checks below)
    if (!s.empty() && s.size() <= 64 && s[0] != '+') {
        double v = 0.0;
        const auto r = std::from_chars(s.data(), s.data() + s.size(), v);
        if (r.ec == std::errc() && r.ptr == s.data() + s.size() && std::isfinite(v)) {
            *out = v;
            return true;
        }
    }
    if (s.empty() || s.size() > 64) {
        if (s.empty()) return false;
        return parse_f64_slow(std::string(s), out);
    }
    size_t i = (s[0] == '+' || s[0] == '-') ? 1 : 0;
    bool digit = false, other = false;
    for (size_t k = i; k < s.size(); ++k) {
        const char c = s[k];
        if (c >= '0' && c <= '9') digit = true;
        else if (!(c == '.' || c == 'e' || c == 'E' || c == '+' || c == '-')) other = true;
    }
    if (other || !digit) return parse_f64_slow(std::string(s), out);  // inf / nan spellings, or invalid
    const char* b = s.data() + (s[0] == '+' ? 1 : 0);
    const char* e = s.data() + s.size();
    if (s[0] == '+' && (b == e || *b == '+' || *b == '-')) return false;
    double v = 0.0;
    const auto r = std::from_chars(b, e, v);
    if (r.ec == std::errc() && r.ptr == e) {
        *out = v;
        return true;
    }
    if (r.ec == std::errc::result_out_of_range) return parse_f64_slow(std::string(s), out);  // inf / 0 like strtod
    return false;
}

static bool parse_f64(const std::string& s, double* out) { return parse_f64_sv(std::string_view(s), out); }

// get_keyword_arguments (parser.rs:879-890): later duplicates win.
using KwArgs = std::unordered_map<std::string, std::pair<bool, std::string>>;  // key -> (has value, value)
static KwArgs keyword_arguments(const std::string& line) {
    KwArgs out;
    auto parts = split(line, ',');
    for (size_t i = 1; i < parts.size(); ++i) {
        const std::string& s = parts[i];
        size_t eq = s.find('=');
        if (eq != std::string::npos) out[trim(s.substr(0, eq))] = {true, trim(s.substr(eq + 1))};
        else out[trim(s)] = {false, std::string()};
    }
    return out;
}
static const std::string* kw_value(const KwArgs& a, const char* key) {
    auto it = a.find(key);
    if (it == a.end() || !it->second.first) return nullptr;
    return &it->second.second;
}

// ------------------------------------------------------------------ model helpers

void Lut::push(double t, double v) {
    data.emplace_back(t, v);
    std::stable_sort(data.begin(), data.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
}

double Lut::interpolate(double temp) const {  // material.rs:36-68
    if (data.size() == 1 || temp <= data[0].first) return data[0].second;
    if (temp >= data.back().first) return data.back().second;
    size_t lo = 0, hi = data.size() - 1;
    while (hi - lo > 1) {
        size_t mid = lo + (hi - lo) / 2;
        if (data[mid].first <= temp) lo = mid;
        else hi = mid;
    }
    double f = (temp - data[lo].first) / (data[hi].first - data[lo].first);
    return data[lo].second + (data[hi].second - data[lo].second) * f;
}

double amplitude_interpolate(double t, const std::vector<double>& ts, const std::vector<double>& vs, double sx,
                             double sy) {  // amplitude.rs:66-98
    if (ts.empty()) return 0.0;
    double tt = t - sx;
    size_t idx = (size_t)(std::lower_bound(ts.begin(), ts.end(), tt) - ts.begin());
    if (idx == 0) return vs.at(0) + sy;
    if (idx >= ts.size()) return vs.at(vs.size() - 1) + sy;
    double t0 = ts[idx - 1], t1 = ts[idx], v0 = vs.at(idx - 1), v1 = vs.at(idx);
    return v0 + (v1 - v0) / (t1 - t0) * (tt - t0) + sy;
}

double Record::eval(const SolverTime& t, int64_t current_step) const {  // amplitude.rs:39-57
    double y;
    if (amp && amp->has_data) {
        y = amplitude_interpolate(amp->total_time ? t.global : t.local, amp->t, amp->v, amp->shift_x, amp->shift_y);
    } else if (current_step > origin_step) {
        y = 1.0;
    } else {
        y = t.local / t.local_max;
    }
    return y * value;
}

// ------------------------------------------------------------------ host workers
// The parser's parallel loops run on worker threads that are started once per process
// (up to 15) and kept, instead of threads started and joined per loop (five loops per
// deck, each paying for its threads' creation). A loop is a job whose tasks are claimed
// through an atomic counter by the calling thread, which always works on its own job,
// and by the workers that take one of its helper entries from the queue; so concurrent
// callers (request-loop slots) share the workers, and a caller finishes its job even
// when no worker is free; a forked child runs its loops on the calling thread alone.
namespace {
struct HostJob {
    std::function<void(size_t)> f;
    size_t ntasks = 0;
    std::atomic<size_t> next{0}, done{0};
    std::mutex m;
    std::condition_variable cv;
    void work() {
        for (size_t t; (t = next.fetch_add(1)) < ntasks;) {
            f(t);
            if (done.fetch_add(1) + 1 == ntasks) {
                std::lock_guard<std::mutex> g(m);
                cv.notify_all();
            }
        }
    }
};

class HostPool {
   public:
    static HostPool& get() {
        static HostPool* p = new HostPool();  // never destroyed: its workers wait on it until exit
        return *p;
    }
    size_t threads() const { return 1 + nworkers_; }
    // f(0 .. ntasks-1), each once, on the caller and up to max_threads - 1 workers
    void run(size_t ntasks, size_t max_threads, std::function<void(size_t)> f) {
        if (ntasks == 0) return;
        if (getpid() != pid_) {  // a forked child: no workers, and the queue's lock may be held
            for (size_t t = 0; t < ntasks; ++t) f(t);
            return;
        }
        auto job = std::make_shared<HostJob>();
        job->f = std::move(f);
        job->ntasks = ntasks;
        const size_t helpers = std::min<size_t>({max_threads, ntasks, threads()}) - 1;
        if (helpers) {
            std::lock_guard<std::mutex> g(m_);
            for (size_t k = 0; k < helpers; ++k) q_.push_back(job);
            cv_.notify_all();
        }
        job->work();
        std::unique_lock<std::mutex> g(job->m);
        job->cv.wait(g, [&] { return job->done.load() == ntasks; });
    }

   private:
    HostPool() : pid_(getpid()) {
        const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
        nworkers_ = hw - 1;
        for (size_t k = 0; k < nworkers_; ++k) std::thread([this] { loop(); }).detach();
    }
    void loop() {
        for (;;) {
            std::shared_ptr<HostJob> job;
            {
                std::unique_lock<std::mutex> g(m_);
                cv_.wait(g, [&] { return !q_.empty(); });
                job = std::move(q_.front());
                q_.pop_front();
            }
            job->work();
        }
    }
    pid_t pid_;
    size_t nworkers_ = 0;
    std::mutex m_;
    std::condition_variable cv_;
    std::deque<std::shared_ptr<HostJob>> q_;
};
}  // namespace

// Runs f(0..ntasks-1), each task once, on up to max_threads threads (the calling thread
// works too; the pool has at most 16).
template <typename F>
static void parallel_tasks(size_t ntasks, F&& f, size_t max_threads = 16) {
    if (ntasks <= 1 || max_threads <= 1) {
        for (size_t t = 0; t < ntasks; ++t) f(t);
        return;
    }
    HostPool::get().run(ntasks, max_threads, std::function<void(size_t)>(std::ref(f)));
}

// ------------------------------------------------------------------ preprocess

// Trimmed, comment-free, upper-cased lines of text[begin, end) (a range of
// whole lines) appended at out + w; a line ending in ',' is joined to the next
// by a space. Returns the new write position.
static size_t preprocess_range(std::string_view text, size_t begin, size_t end, char* out, size_t w) {
    size_t start = begin;
    while (start < end) {
        const void* hit = std::memchr(text.data() + start, '\n', end - start);
        const size_t nl = hit ? (size_t)((const char*)hit - text.data()) : end;
        size_t a = start, b = nl;
        while (a < b && is_ws(text[a])) ++a;
        while (b > a && is_ws(text[b - 1])) --b;
        if (a < b && !(b - a >= 2 && text[a] == '*' && text[a + 1] == '*')) {
            const char* src = text.data() + a;
            char* dst = out + w;
            const size_t len = b - a;
            for (size_t k = 0; k < len; ++k) {  // ASCII to_uppercase (a loop the compiler vectorises)
                const char c = src[k];
                dst[k] = (c >= 'a' && c <= 'z') ? (char)(c - 'a' + 'A') : c;
            }
            w += len;
            out[w++] = text[b - 1] == ',' ? ' ' : '\n';
        }
        start = nl + 1;
    }
    return w;
}

// substitute_ccx_solvers (parser.rs:930-942)
static const char* const kSolverPats[] = {"ITERATIVE CHOLESKY", "ITERATIVE SCALING", "PASTIX", "PARDISO", "SPOOLES"};
static const char* const kSolverReps[] = {"ITERATIVE", "ITERATIVE", "DIRECT", "DIRECT", "DIRECT"};

// Replaces the solver names in buf[0, len) in place in one left-to-right pass
// over non-overlapping matches, as aho-corasick's replace_all does (standard
// semantics; these five names never overlap or contain one another, so that is
// the leftmost match at each point, and a replacement never forms a new match:
// "ITERATIVE CHOLESKY SCALING" becomes "ITERATIVE SCALING"). No replacement is
// longer than its name. Returns the new length.
static size_t substitute_solvers(char* buf, size_t len) {
    bool any = false;
    for (const char* q : kSolverPats)
        if (std::string_view(buf, len).find(q) != std::string_view::npos) any = true;
    if (!any) return len;
    size_t r = 0, w = 0;
    while (r < len) {
        int hit = -1;
        const char c = buf[r];
        if (c == 'I' || c == 'P' || c == 'S')
            for (int k = 0; k < 5 && hit < 0; ++k) {
                const size_t pl = std::strlen(kSolverPats[k]);
                if (len - r >= pl && std::memcmp(buf + r, kSolverPats[k], pl) == 0) hit = k;
            }
        if (hit < 0) {
            buf[w++] = buf[r++];
            continue;
        }
        const size_t rl = std::strlen(kSolverReps[hit]);
        std::memmove(buf + w, kSolverReps[hit], rl);
        w += rl;
        r += std::strlen(kSolverPats[hit]);
    }
    return w;
}

// Writes the str::lines views of text[a, b) (trailing '\r' dropped) to
// lines[0..) and appends first + (index) of every keyword line ('*') to kw.
static void split_lines(const char* text, size_t a, size_t b, std::string_view* lines, size_t first,
                        std::vector<size_t>& kw) {
    size_t k = 0;
    while (a < b) {
        const void* hit = std::memchr(text + a, '\n', b - a);
        const size_t end = hit ? (size_t)((const char*)hit - text) : b;
        size_t e2 = end;
        if (e2 > a && text[e2 - 1] == '\r') --e2;
        if (e2 > a && text[a] == '*') kw.push_back(first + k);
        lines[k++] = std::string_view(text + a, e2 - a);
        a = end + 1;
    }
}

static size_t count_lines(const char* text, size_t a, size_t b) {
    size_t k = 0;
    while (a < b) {
        const void* hit = std::memchr(text + a, '\n', b - a);
        ++k;
        if (!hit) break;
        a = (size_t)((const char*)hit - text) + 1;
    }
    return k;
}

// True when the input line ending at the newline `nl` is kept by the
// preprocessor (not blank, not a comment) and does not end in ',' (so no
// logical line continues past it).
static bool ends_logical_line(std::string_view text, size_t lo, size_t nl) {
    size_t a = nl;
    while (a > lo && text[a - 1] != '\n') --a;
    size_t b = nl;
    while (a < b && is_ws(text[a])) ++a;
    while (b > a && is_ws(text[b - 1])) --b;
    if (a == b) return false;
    if (b - a >= 2 && text[a] == '*' && text[a + 1] == '*') return false;
    return text[b - 1] != ',';
}

// Lines of the preprocessed text (parser.rs:903-942 followed by str::lines) as
// views into `store`. The input is cut into chunks only after lines that end a
// logical line, so every output line, and every solver name, lies inside one
// chunk: each thread preprocesses its chunk into its own region of `store`,
// substitutes the solver names there, and then indexes that region's lines.
static void preprocess_lines(std::string_view text, std::unique_ptr<char[]>& store,
                             std::vector<std::string_view>& lines, std::vector<size_t>& keyword_lines) {
    const size_t n = text.size();
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const size_t nthreads = std::min<size_t>(hw, std::max<size_t>(1, n / (1u << 20)));
    std::vector<size_t> cut(nthreads + 1, n);
    cut[0] = 0;
    for (size_t t = 1; t < nthreads; ++t) {
        size_t c = std::max(cut[t - 1], n * t / nthreads);
        cut[t] = n;
        while (c < n) {
            const void* hit = std::memchr(text.data() + c, '\n', n - c);
            if (!hit) break;
            const size_t nl = (size_t)((const char*)hit - text.data());
            if (ends_logical_line(text, cut[t - 1], nl)) {
                cut[t] = nl + 1;
                break;
            }
            c = nl + 1;
        }
    }
    store.reset(new char[n + 1]);  // a chunk's output is never longer than its input (+1 for the last)
    char* out = store.get();
    std::vector<size_t> len(nthreads, 0), nlines(nthreads, 0), first(nthreads + 1, 0);
    auto run = [&](auto&& fn) { parallel_tasks(nthreads, fn, nthreads); };
    run([&](size_t t) {
        len[t] = preprocess_range(text, cut[t], cut[t + 1], out, cut[t]) - cut[t];
        len[t] = substitute_solvers(out + cut[t], len[t]);
        nlines[t] = count_lines(out, cut[t], cut[t] + len[t]);
    });
    for (size_t t = 0; t < nthreads; ++t) first[t + 1] = first[t] + nlines[t];
    lines.resize(first[nthreads]);
    std::vector<std::vector<size_t>> kw(nthreads);
    run([&](size_t t) { split_lines(out, cut[t], cut[t] + len[t], lines.data() + first[t], first[t], kw[t]); });
    keyword_lines.clear();
    for (auto& v : kw) keyword_lines.insert(keyword_lines.end(), v.begin(), v.end());
}

// ------------------------------------------------------------------ parser

namespace {

const std::unordered_set<std::string>& keywords() {
    static const std::unordered_set<std::string> k = {
        "NODE", "ELEMENT", "NSET", "ELSET", "MATERIAL", "ELASTIC", "DENSITY", "SOLID_SECTION", "STEP", "STATIC",
        "BOUNDARY", "CLOAD", "END_STEP", "HEADING", "NODE_FILE", "EL_FILE", "AMPLITUDE", "SURFACE", "DLOAD",
        "DSLOAD", "NODE_PRINT", "EL_PRINT", "INCLUDE", "BEAM_SECTION", "EXPANSION", "SHELL_SECTION",
        "CONDUCTIVITY", "SPECIFIC_HEAT", "INITIAL_CONDITIONS", "DEPVAR"};
    return k;
}

// Data blocks of *NODE and *ELEMENT (TYPE=C3D4 / C3D20), parsed ahead of the
// keyword state machine by several threads. The state machine then applies a
// block's rows in line order, exactly as it would apply the lines one by one; a
// block with any line that does not parse is left to the line-by-line path,
// which reports the error as before.
struct PreBlock {
    size_t begin = 0, end = 0;  // line range of the data lines
    int npe = 0;                // 0: *NODE, 4 / 20: *ELEMENT of that type
    bool ok = true;
    RawVec<int64_t> ids;
    RawVec<std::array<double, 3>> xyz;  // *NODE
    RawVec<int64_t> conn;               // *ELEMENT: npe per line
};

// Parses every block's lines into its arrays: tasks of up to 2,048 lines of
// any block, taken in turn by up to 16 threads (each writes only its lines'
// slots). A block with a line that does not parse is marked not ok.
static void preparse_blocks(const std::vector<std::string_view>& lines, std::vector<PreBlock>& blocks) {
    constexpr size_t kTask = 2048;
    struct Task {
        size_t block, a, e;
    };
    std::vector<Task> tasks;
    for (size_t bi = 0; bi < blocks.size(); ++bi) {
        PreBlock& b = blocks[bi];
        const size_t n = b.end - b.begin;
        b.ids.resize(n);
        if (b.npe == 0) b.xyz.resize(n);
        else b.conn.resize((size_t)b.npe * n);
        for (size_t a = 0; a < n; a += kTask) tasks.push_back({bi, a, std::min(n, a + kTask)});
    }
    std::vector<uint8_t> bad(tasks.size(), 0);
    parallel_tasks(tasks.size(), [&](size_t ti) {
        std::vector<std::string_view> f;
        f.reserve(24);
        const Task& t = tasks[ti];
        PreBlock& b = blocks[t.block];
        for (size_t k = t.a; k < t.e; ++k) {
            const std::string_view line = lines[b.begin + k];
            size_t s = 0, z = line.size();
            while (s < z && is_ws(line[s])) ++s;
            if (s == z) {  // blank lines are skipped by the state machine: keep the block exact
                bad[ti] = 1;
                return;
            }
            split_views(line, ',', f);
            bool ok;
            if (b.npe == 0) {
                ok = f.size() == 4 && parse_usize_sv(f[0], &b.ids[k]) && parse_f64_sv(f[1], &b.xyz[k][0]) &&
                     parse_f64_sv(f[2], &b.xyz[k][1]) && parse_f64_sv(f[3], &b.xyz[k][2]);
            } else {
                ok = (int)f.size() == b.npe + 1 && parse_usize_sv(f[0], &b.ids[k]);
                for (int a2 = 0; ok && a2 < b.npe; ++a2) ok = parse_usize_sv(f[a2 + 1], &b.conn[(size_t)b.npe * k + a2]);
            }
            if (!ok) {
                bad[ti] = 1;
                return;
            }
        }
    });
    for (size_t ti = 0; ti < tasks.size(); ++ti)
        if (bad[ti]) blocks[tasks[ti].block].ok = false;
}

struct Parser {
    // Lines of the preprocessed text as views; a line becomes a std::string only
    // when the state machine reads it (not for pre-parsed *NODE / *ELEMENT blocks).
    std::unique_ptr<char[]> store;
    std::vector<std::string_view> views;
    std::unordered_map<size_t, std::string> cache;  // references stay valid as it grows
    const std::string& line_at(size_t i) {
        auto it = cache.find(i);
        if (it == cache.end()) it = cache.emplace(i, std::string(views[i])).first;
        return it->second;
    }
    std::vector<PreBlock> blocks;  // sorted by begin
    size_t next_block = 0;
    size_t pos = 0;
    Project p;
    std::string kw;  // current keyword ("" = none)
    int64_t line_nr = 0;
    bool has_elem_type = false, has_elset = false, has_set = false, is_generate = false;
    std::string elem_type, elset_name, set_name;
    bool in_step = false;
    StaticStep cur;
    int64_t step_counter = 0;
    std::vector<Record> step_loads, step_bcs;
    bool has_ic = false;
    std::string ic_type;

    [[noreturn]] void perr(const std::string& msg) {
        fail_detail(FX_PARSE, "Parsing error at line " + std::to_string(line_nr) + ": " + msg, (int64_t)line_nr, -1,
                    msg);
    }
    const std::string* peek() { return pos < views.size() ? &line_at(pos) : nullptr; }

    void finish_step() {
        cur.loads = step_loads;
        cur.bcs = step_bcs;
        p.steps.push_back(cur);
        in_step = false;
        cur = StaticStep();
    }

    std::vector<int64_t> targets(const std::string& t0) {
        std::string t = trim(t0);
        auto it = p.node_sets.find(t);
        if (it != p.node_sets.end()) return it->second;
        int64_t id;
        if (parse_usize(t, &id)) return {id};
        return {};
    }

    std::shared_ptr<const Amplitude> amp_for(const std::string* name) {
        if (!name) return nullptr;
        auto it = p.amplitudes.find(*name);
        return it == p.amplitudes.end() ? nullptr : it->second;
    }

    int64_t origin() const { return in_step ? step_counter : 0; }

    // Applies a pre-parsed block if the state machine is in the matching keyword
    // (what data() would do line by line); false = parse the lines one by one.
    bool apply_block(PreBlock& b) {
        if (b.npe == 0) {
            if (kw != "NODE") return false;
            if (p.node_line_ids.empty()) {  // the usual single *NODE block: take the arrays
                p.node_line_ids.swap(b.ids);
                p.node_line_xyz.swap(b.xyz);
            } else {
                p.node_line_ids.insert(p.node_line_ids.end(), b.ids.begin(), b.ids.end());
                p.node_line_xyz.insert(p.node_line_xyz.end(), b.xyz.begin(), b.xyz.end());
            }
            return true;
        }
        if (kw != "ELEMENT" || !has_elem_type) return false;
        if (!((b.npe == 4 && elem_type == "C3D4") || (b.npe == 20 && elem_type == "C3D20"))) return false;
        if (has_elset && !elset_name.empty()) {
            auto& eset = p.element_sets[elset_name];
            eset.insert(eset.end(), b.ids.begin(), b.ids.end());
        }
        const int64_t off0 = (int64_t)p.elem_line_conn.size();
        const size_t m = b.ids.size(), at = p.elem_line_off.size();
        p.elem_line_npe.insert(p.elem_line_npe.end(), m, (uint8_t)b.npe);
        p.elem_line_off.resize(at + m);
        for (size_t k = 0; k < m; ++k) p.elem_line_off[at + k] = off0 + (int64_t)(b.npe * k);
        if (p.elem_line_ids.empty()) {  // the first bulk *ELEMENT block: take the arrays
            p.elem_line_ids.swap(b.ids);
            p.elem_line_conn.swap(b.conn);
        } else {
            p.elem_line_ids.insert(p.elem_line_ids.end(), b.ids.begin(), b.ids.end());
            p.elem_line_conn.insert(p.elem_line_conn.end(), b.conn.begin(), b.conn.end());
        }
        return true;
    }

    void run() {
        while (pos < views.size()) {
            line_nr = (int64_t)pos + 1;
            while (next_block < blocks.size() && blocks[next_block].begin < pos) ++next_block;
            if (next_block < blocks.size() && blocks[next_block].begin == pos && blocks[next_block].ok &&
                apply_block(blocks[next_block])) {
                pos = blocks[next_block].end;
                ++next_block;
                continue;
            }
            const std::string& line = line_at(pos++);
            if (!line.empty() && line[0] == '*') {
                keyword(line);
                continue;
            }
            if (line.empty() || kw.empty()) continue;
            if (!is_ws(line.front()) && !is_ws(line.back())) {  // already trimmed (the usual case)
                data(line);
                continue;
            }
            std::string t = trim(line);
            if (t.empty()) continue;
            data(t);
        }
        if (in_step) finish_step();
        p.resolve_mesh();
    }

    void keyword(const std::string& line) {
        auto parts = split(line, ',');
        std::string k0 = trim(parts[0]);
        std::string name = trim(k0.substr(1));
        for (auto& c : name) c = (char)std::toupper((unsigned char)c);
        std::string key = name;
        std::replace(key.begin(), key.end(), ' ', '_');
        if (!keywords().count(key))
            fail_detail(FX_UNSUPPORTED_KEYWORD, "Unsupported keyword at line " + std::to_string(line_nr) + ": " + name,
                        (int64_t)line_nr, -1, name);
        kw = key;
        KwArgs ka = keyword_arguments(line);
        if (key == "ELEMENT") {
            const std::string* t = kw_value(ka, "TYPE");
            has_elem_type = t != nullptr;
            elem_type = t ? *t : "";
            const std::string* es = kw_value(ka, "ELSET");
            has_elset = es != nullptr;
            elset_name = es ? *es : "";
        } else if (key == "NSET" || key == "ELSET") {
            const std::string* s = kw_value(ka, key.c_str());
            has_set = s != nullptr;
            set_name = s ? *s : "";
            is_generate = ka.count("GENERATE") > 0;
        } else if (key == "MATERIAL") {
            const std::string* n = kw_value(ka, "NAME");
            if (!n) perr("Material name not found");
            Material m;
            m.name = *n;
            p.materials.push_back(m);
        } else if (key == "EXPANSION") {
            if (!p.materials.empty()) {
                const std::string* z = kw_value(ka, "ZERO");
                if (z) {
                    double v;
                    if (!parse_f64(*z, &v)) perr("Invalid ZERO value in *EXPANSION");
                    p.materials.back().tref = v;
                }
            }
        } else if (key == "INITIAL_CONDITIONS") {
            const std::string* t = kw_value(ka, "TYPE");
            has_ic = t != nullptr;
            ic_type = t ? *t : "";
            for (auto& c : ic_type) c = (char)std::toupper((unsigned char)c);
        } else if (key == "SOLID_SECTION") {
            const std::string* es = kw_value(ka, "ELSET");
            if (!es) perr("Elset not found in *SOLID SECTION");
            const std::string* mn = kw_value(ka, "MATERIAL");
            if (!mn) perr("Material not found in *SOLID SECTION");
            int midx = -1;
            for (size_t i = 0; i < p.materials.size(); ++i)
                if (p.materials[i].name == *mn) {
                    midx = (int)i;
                    break;
                }
            if (midx < 0) fail_detail(FX_MATERIAL_NOT_FOUND, "Material " + *mn + " not found", -1, -1, *mn);
            auto it = p.element_sets.find(*es);
            if (it == p.element_sets.end()) fail_detail(FX_ELSET_NOT_FOUND, "Elset " + *es + " not found", -1, -1, *es);
            for (int64_t eid : it->second) p.elem_material_lines.emplace_back(eid, midx);
        } else if (key == "STEP") {
            if (step_counter == 0) {
                step_loads = p.initial_loads;
                step_bcs = p.initial_bcs;
            }
            step_counter += 1;
            if (in_step) finish_step();
            bool nlgeom = ka.count("NLGEOM") > 0;
            int64_t max_inc = 10000;
            const std::string* inc = kw_value(ka, "INC");
            if (inc) {
                int64_t v;
                if (parse_usize(*inc, &v)) max_inc = v;
            }
            const std::string* nxt = peek();
            if (nxt && starts_with(*nxt, "*STATIC")) {
                KwArgs ska = keyword_arguments(*nxt);
                const std::string* sv = kw_value(ska, "SOLVER");
                SolverType st = SolverType::Default;
                if (sv) {
                    if (*sv == "DIRECT") st = SolverType::Direct;
                    else if (*sv == "ITERATIVE") st = SolverType::Iterative;
                    else fail_detail(FX_UNKNOWN_SOLVER, "Unknown solver type: " + *sv, -1, -1, *sv);
                }
                ++pos;  // consume *STATIC
                IncrementData incd;
                incd.max_increments = max_inc;
                const std::string* dl = peek();
                if (dl && !starts_with(*dl, "*")) {
                    auto args = split(*dl, ',');
                    for (auto& a : args) a = trim(a);
                    if (args.size() >= 4) {
                        if (!parse_f64(args[0], &incd.initial)) perr("Invalid initial time increment");
                        if (!parse_f64(args[1], &incd.period)) perr("Invalid time period");
                        if (!parse_f64(args[2], &incd.min_inc)) perr("Invalid min time increment");
                        if (!parse_f64(args[3], &incd.max_inc)) perr("Invalid max time increment");
                    }
                    ++pos;  // consume the data line
                }
                cur = StaticStep();
                cur.solver = st;
                cur.inc = incd;
                cur.nlgeom = nlgeom;
                in_step = true;
            }
        } else if (key == "END_STEP") {
            if (in_step) finish_step();
        } else if (key == "AMPLITUDE") {
            const std::string* n = kw_value(ka, "NAME");
            if (!n) perr("Amplitude card is missing a Name= argument");
            auto a = std::make_shared<Amplitude>();
            const std::string* tt = kw_value(ka, "TIME");
            a->total_time = tt && *tt == "TOTAL TIME";
            double v;
            const std::string* sx = kw_value(ka, "SHIFTX");
            if (sx && parse_f64(*sx, &v)) a->shift_x = v;
            const std::string* sy = kw_value(ka, "SHIFTY");
            if (sy && parse_f64(*sy, &v)) a->shift_y = v;
            const std::string* nxt = peek();
            if (nxt) {
                auto f = split(*nxt, ',');
                for (size_t i = 0; i < f.size(); i += 2) {
                    double x;
                    if (parse_f64(trim(f[i]), &x)) a->t.push_back(x);
                }
                for (size_t i = 1; i < f.size(); i += 2) {
                    double x;
                    if (!parse_f64(trim(f[i]), &x)) perr("Invalid amplitude value");
                    a->v.push_back(x);
                }
                a->has_data = true;
                p.amplitudes[*n] = a;
            }
        } else if (key == "BOUNDARY") {
            const std::string* an = kw_value(ka, "AMPLITUDE");
            std::string amp_name = an ? *an : "";
            const std::string* op = kw_value(ka, "OP");
            if (op && *op == "NEW") {
                if (in_step) step_bcs.clear();
                else p.initial_bcs.clear();
            }
            const std::string* nxt = peek();
            if (nxt && !starts_with(*nxt, "*")) boundary(*nxt, an ? &amp_name : nullptr);
        } else if (key == "CLOAD") {
            const std::string* an = kw_value(ka, "AMPLITUDE");
            std::string amp_name = an ? *an : "";
            const std::string* op = kw_value(ka, "OP");
            if (op && *op == "NEW") {
                if (in_step) step_loads.clear();
                else p.initial_loads.clear();
            }
            while (const std::string* nxt = peek()) {
                if (starts_with(*nxt, "*")) break;
                std::string l = *nxt;
                ++pos;
                cload(l, an ? &amp_name : nullptr);
            }
        }
    }

    void cload(const std::string& line, const std::string* amp) {  // parser.rs:740-798
        auto parts = split(line, ',');
        for (auto& s : parts) s = trim(s);
        if (parts.size() < 3) return;
        int64_t dof;
        if (!parse_usize(parts[1], &dof)) perr("Invalid DOF");
        double val;
        if (!parse_f64(parts[2], &val)) perr("Invalid load value");
        auto nodes = targets(parts[0]);
        if (dof >= 1 && dof <= 3) {
            for (int64_t nid : nodes) {
                Record r{nid, (int)(dof - 1), val, amp_for(amp), origin()};
                (in_step ? step_loads : p.initial_loads).push_back(r);
            }
        }
    }

    void boundary(const std::string& line, const std::string* amp) {  // parser.rs:800-876
        auto parts = split(line, ',');
        for (auto& s : parts) s = trim(s);
        if (parts.size() < 2) return;
        int64_t first, last;
        if (!parse_usize(parts[1], &first)) perr("Invalid first DOF");
        if (parts.size() > 2 && !parts[2].empty()) {
            if (!parse_usize(parts[2], &last)) perr("Invalid last DOF");
        } else {
            last = first;
        }
        double val = 0.0;
        if (parts.size() > 3 && !parse_f64(parts[3], &val)) perr("Invalid boundary value");
        for (int64_t nid : targets(parts[0]))
            for (int64_t d = first; d <= last; ++d)
                if (d >= 1 && d <= 3) {
                    Record r{nid, (int)(d - 1), val, amp_for(amp), origin()};
                    (in_step ? step_bcs : p.initial_bcs).push_back(r);
                }
    }

    std::vector<std::string_view> fields;  // reused by the bulk data lines

    void data(const std::string& line) {
        if (kw == "NODE") {
            split_views(line, ',', fields);
            int64_t id;
            std::array<double, 3> x;
            if (fields.size() != 4 || !parse_usize_sv(fields[0], &id) || !parse_f64_sv(fields[1], &x[0]) ||
                !parse_f64_sv(fields[2], &x[1]) || !parse_f64_sv(fields[3], &x[2]))
                perr("Invalid node definition: " + line);
            p.node_line_ids.push_back(id);
            p.node_line_xyz.push_back(x);
        } else if (kw == "ELEMENT") {
            if (!has_elem_type) return;
            split_views(line, ',', fields);
            std::vector<int64_t> nums;
            nums.reserve(fields.size());
            for (auto s : fields) {
                int64_t v;
                if (!parse_usize_sv(s, &v))
                    fail_detail(FX_PARSE, "Parsing error at line 0: Integer conversion failed", 0, -1,
                                "Integer conversion failed");
                nums.push_back(v);
            }
            int npe;
            if (elem_type == "C3D4") npe = 4;
            else if (elem_type == "C3D20") npe = 20;
            else
                fail_detail(FX_PARSE, "Parsing error at line 0: Unknown element definition: " + elem_type, 0, -1,
                            "Unknown element definition: " + elem_type);
            if ((int)nums.size() - 1 != npe)
                fail_detail(FX_PARSE, "Parsing error at line 0: Wrong node count for " + elem_type, 0, -1,
                            "Wrong node count for " + elem_type);
            int64_t eid = nums[0];
            if (has_elset && !elset_name.empty()) p.element_sets[elset_name].push_back(eid);
            p.elem_line_ids.push_back(eid);
            p.elem_line_npe.push_back((uint8_t)npe);
            p.elem_line_off.push_back((int64_t)p.elem_line_conn.size());
            p.elem_line_conn.insert(p.elem_line_conn.end(), nums.begin() + 1, nums.end());
        } else if (kw == "NSET" || kw == "ELSET") {
            if (!has_set || is_generate) return;
            std::vector<int64_t> ids;
            for (auto& s : split(line, ',')) {
                std::string t = trim(s);
                int64_t v;
                if (!t.empty() && parse_usize(t, &v)) ids.push_back(v);
            }
            if (kw == "NSET") {
                auto& dst = p.node_sets[set_name];
                dst.insert(dst.end(), ids.begin(), ids.end());
            } else if (line.find(',') == std::string::npos && ids.empty()) {
                auto it = p.element_sets.find(trim(line));
                if (it != p.element_sets.end()) {
                    std::vector<int64_t> add = it->second;
                    auto& dst = p.element_sets[set_name];
                    dst.insert(dst.end(), add.begin(), add.end());
                }
            } else {
                auto& dst = p.element_sets[set_name];
                dst.insert(dst.end(), ids.begin(), ids.end());
            }
        } else if (kw == "ELASTIC" || kw == "DENSITY" || kw == "EXPANSION") {
            if (p.materials.empty()) return;
            std::vector<double> v;
            for (auto& s : split(line, ',')) {
                double x;
                if (!parse_f64(trim(s), &x)) {
                    if (kw == "ELASTIC") perr("Invalid elastic constant");
                    if (kw == "DENSITY") perr("Invalid density value");
                    perr("Invalid expansion constant");
                }
                v.push_back(x);
            }
            Material& m = p.materials.back();
            if (kw == "ELASTIC") {
                if (v.size() >= 2) {
                    double t = v.size() >= 3 ? v[2] : 0.0;
                    m.e.push(t, v[0]);
                    m.has_e = true;
                    m.nu.push(t, v[1]);
                    m.has_nu = true;
                }
            } else if (!v.empty()) {
                double t = v.size() >= 2 ? v[1] : 0.0;
                if (kw == "DENSITY") { m.density.push(t, v[0]); m.has_density = true; }
                else { m.alpha.push(t, v[0]); m.has_alpha = true; }
            }
        } else if (kw == "INITIAL_CONDITIONS") {
            if (!has_ic || ic_type != "TEMPERATURE") return;
            auto parts = split(line, ',');
            for (auto& s : parts) s = trim(s);
            if (parts.size() >= 2) {
                double t;
                if (!parse_f64(parts[1], &t)) perr("Invalid temperature value");
                for (int64_t nid : targets(parts[0])) p.initial_temperatures[nid] = t;
            }
        } else if (kw == "DEPVAR") {
            if (p.materials.empty()) return;
            auto parts = split(line, ',');
            int64_t n;
            if (!parse_usize(trim(parts[0]), &n)) perr("Invalid DEPVAR value");
            p.materials.back().depvars = n;
        } else if (kw == "NODE_FILE" || kw == "EL_FILE") {
            auto& dst = kw == "NODE_FILE" ? p.nodal_output : p.element_output;
            for (auto& s : split(line, ',')) dst.push_back(trim(s));
        }
    }
};

}  // namespace

Project parse_inp(std::string_view text) {
    Parser ps;
    std::vector<size_t> kwl;  // indices of the keyword lines
    preprocess_lines(text, ps.store, ps.views, kwl);
    // *NODE / *ELEMENT data blocks: keyword line followed by data lines up to the next keyword
    const auto& V = ps.views;
    for (size_t q = 0; q < kwl.size(); ++q) {
        const size_t i = kwl[q];
        const std::string_view l = V[i];
        const size_t e = q + 1 < kwl.size() ? kwl[q + 1] : V.size();
        if (e - i - 1 < 1024) continue;  // small blocks: line by line
        const std::string kl(l);
        std::string name = trim(kl.substr(1, kl.find(',') == std::string::npos ? std::string::npos : kl.find(',') - 1));
        std::replace(name.begin(), name.end(), ' ', '_');
        PreBlock b;
        b.begin = i + 1;
        b.end = e;
        if (name == "NODE") {
            b.npe = 0;
        } else if (name == "ELEMENT") {
            KwArgs ka = keyword_arguments(kl);
            const std::string* t = kw_value(ka, "TYPE");
            if (!t || (*t != "C3D4" && *t != "C3D20")) continue;
            b.npe = *t == "C3D4" ? 4 : 20;
        } else {
            continue;
        }
        ps.blocks.push_back(std::move(b));
    }
    preparse_blocks(ps.views, ps.blocks);
    ps.run();
    return std::move(ps.p);
}

void IdIndex::build(const std::vector<int64_t>& ids) {
    table.clear();
    map.clear();
    count = (int64_t)ids.size();
    base = ids.empty() ? 0 : ids.front();
    if (ids.empty() || ids.back() - base == count - 1) {  // ascending and unique: consecutive
        mode = 0;
        return;
    }
    const int64_t span = ids.back() - base + 1;
    if (span <= 8 * count + 4096) {
        mode = 1;
        table.assign((size_t)span, -1);
        for (int64_t i = 0; i < count; ++i) table[(size_t)(ids[(size_t)i] - base)] = (int32_t)i;
        return;
    }
    mode = 2;
    map.reserve((size_t)count);
    for (int64_t i = 0; i < count; ++i) map[ids[(size_t)i]] = i;
}

// Ascending unique ids of `line_ids` with, for each, the last line that defines
// it (what repeated map inserts in line order leave behind).
static void last_definitions(const RawVec<int64_t>& line_ids, std::vector<int64_t>& ids,
                             std::vector<int64_t>& line) {
    const size_t n = line_ids.size();
    bool ascending = true;
    for (size_t i = 1; i < n && ascending; ++i) ascending = line_ids[i] > line_ids[i - 1];
    ids.clear();
    line.clear();
    if (ascending) {
        ids.assign(line_ids.begin(), line_ids.end());
        line.resize(n);
        for (size_t i = 0; i < n; ++i) line[i] = (int64_t)i;
        return;
    }
    std::vector<int64_t> perm(n);
    for (size_t i = 0; i < n; ++i) perm[i] = (int64_t)i;
    std::stable_sort(perm.begin(), perm.end(), [&](int64_t a, int64_t b) { return line_ids[a] < line_ids[b]; });
    ids.reserve(n);
    line.reserve(n);
    for (size_t k = 0; k < n; ++k) {
        const int64_t id = line_ids[(size_t)perm[k]];
        if (!ids.empty() && ids.back() == id) line.back() = perm[k];  // a later line of the same id
        else {
            ids.push_back(id);
            line.push_back(perm[k]);
        }
    }
}

void Project::resolve_mesh() {
    std::vector<int64_t> nline;
    last_definitions(node_line_ids, index_to_node_id, nline);
    node_xyz.resize(nline.size());
    if (nline.size() == node_line_xyz.size()) node_xyz.swap(node_line_xyz);  // no repeats: identity
    else
        for (size_t i = 0; i < nline.size(); ++i) node_xyz[i] = node_line_xyz[(size_t)nline[i]];
    node_index.build(index_to_node_id);
    last_definitions(elem_line_ids, elem_ids, elem_line);
}

DenseModel build_dense(const Project& p) {
    DenseModel d;
    d.n_nodes = p.n_nodes();
    d.xyz.resize(3 * d.n_nodes);
    if (d.n_nodes) std::memcpy(d.xyz.data(), p.node_xyz.data(), d.xyz.size() * sizeof(double));
    // material of every element (ascending id order): the last assignment wins
    const int64_t ne = p.n_elements();
    IdIndex eindex;
    eindex.build(p.elem_ids);
    std::vector<int32_t> mat((size_t)ne, -1);
    for (const auto& em : p.elem_material_lines) {
        const int64_t k = eindex.find(em.first);
        if (k >= 0) mat[(size_t)k] = em.second;
    }
    d.g4.npe = 4;
    d.g20.npe = 20;
    // each element's slot in its group (ascending id within the group)
    std::vector<int32_t> slot((size_t)ne);
    int64_t n4 = 0, n20 = 0;
    for (int64_t k = 0; k < ne; ++k)
        slot[(size_t)k] = (int32_t)(p.elem_line_npe[(size_t)p.elem_line[(size_t)k]] == 4 ? n4++ : n20++);
    for (ElemGroup* g : {&d.g4, &d.g20}) {
        const int64_t m = g == &d.g4 ? n4 : n20;
        g->elem_ids.resize((size_t)m);
        g->conn.resize((size_t)m * g->npe);
        g->mat.resize((size_t)m);
    }
    // connectivity as node indices, in tasks of 2,048 elements; the first unknown
    // node in element order is the one reported (NodeNotFound)
    constexpr int64_t kTask = 2048;
    const size_t ntask = (size_t)((ne + kTask - 1) / kTask);
    std::vector<int64_t> miss_k(ntask, -1), miss_id(ntask, 0);
    parallel_tasks(ntask, [&](size_t t) {
        for (int64_t k = (int64_t)t * kTask; k < std::min<int64_t>(ne, ((int64_t)t + 1) * kTask); ++k) {
            const size_t line = (size_t)p.elem_line[(size_t)k];
            const int npe = p.elem_line_npe[line];
            ElemGroup& g = npe == 4 ? d.g4 : d.g20;
            const size_t pos = (size_t)slot[(size_t)k];
            g.elem_ids[pos] = p.elem_ids[(size_t)k];
            g.mat[pos] = mat[(size_t)k];
            const int64_t* nodes = &p.elem_line_conn[(size_t)p.elem_line_off[line]];
            int32_t* c = &g.conn[pos * (size_t)npe];
            for (int a = 0; a < npe; ++a) {
                const int64_t idx = p.index_of(nodes[a]);
                if (idx < 0 && miss_k[t] < 0) {
                    miss_k[t] = k;
                    miss_id[t] = nodes[a];
                }
                c[a] = (int32_t)(idx < 0 ? 0 : idx);
            }
        }
    });
    for (size_t t = 0; t < ntask; ++t)
        if (miss_k[t] >= 0) {
            d.missing_node_id = miss_id[t];
            d.missing_node_error = "Node " + std::to_string(miss_id[t]) + " not found in mesh";
            break;
        }
    // mesh volume: tets exactly; bricks as 6 Kuhn tets of their 8 corner nodes. The
    // tet volumes are computed in parallel and summed in element order on one thread.
    auto tet_vol = [&](int a, int b, int c, int e) {
        const double* A = &d.xyz[3 * (size_t)a];
        const double* B = &d.xyz[3 * (size_t)b];
        const double* Cc = &d.xyz[3 * (size_t)c];
        const double* E = &d.xyz[3 * (size_t)e];
        double u[3], v[3], w[3];
        for (int k = 0; k < 3; ++k) {
            u[k] = B[k] - A[k];
            v[k] = Cc[k] - A[k];
            w[k] = E[k] - A[k];
        }
        return std::fabs(u[0] * (v[1] * w[2] - v[2] * w[1]) - u[1] * (v[0] * w[2] - v[2] * w[0]) +
                         u[2] * (v[0] * w[1] - v[1] * w[0])) / 6.0;
    };
    static const int kuhn[6][4] = {{0, 1, 2, 6}, {0, 2, 3, 6}, {0, 3, 7, 6}, {0, 7, 4, 6}, {0, 4, 5, 6}, {0, 5, 1, 6}};
    RawVec<double> tv((size_t)(n4 + 6 * n20));
    const size_t vt4 = (size_t)((n4 + kTask - 1) / kTask), vt20 = (size_t)((n20 + kTask - 1) / kTask);
    parallel_tasks(vt4 + vt20, [&](size_t t) {
        if (t < vt4) {
            for (int64_t e = (int64_t)t * kTask; e < std::min<int64_t>(n4, ((int64_t)t + 1) * kTask); ++e) {
                const int32_t* c = &d.g4.conn[4 * (size_t)e];
                tv[(size_t)e] = tet_vol(c[0], c[1], c[2], c[3]);
            }
        } else {
            const int64_t t20 = (int64_t)(t - vt4);
            for (int64_t e = t20 * kTask; e < std::min<int64_t>(n20, (t20 + 1) * kTask); ++e) {
                const int32_t* c = &d.g20.conn[20 * (size_t)e];
                for (int q = 0; q < 6; ++q)
                    tv[(size_t)(n4 + 6 * e + q)] = tet_vol(c[kuhn[q][0]], c[kuhn[q][1]], c[kuhn[q][2]], c[kuhn[q][3]]);
            }
        }
    });
    for (double v : tv) d.volume += v;
    MatTableHost& m = d.mats;
    for (const Material& mat : p.materials) {
        auto add = [&](bool has, const Lut& l, std::vector<int32_t>& off, std::vector<int32_t>& len) {
            off.push_back((int32_t)m.t.size());
            len.push_back(has ? (int32_t)l.data.size() : 0);
            if (has)
                for (auto& tv : l.data) {
                    m.t.push_back(tv.first);
                    m.v.push_back(tv.second);
                }
        };
        add(mat.has_e, mat.e, m.e_off, m.e_len);
        add(mat.has_nu, mat.nu, m.nu_off, m.nu_len);
        add(mat.has_alpha, mat.alpha, m.a_off, m.a_len);
        m.tref.push_back(mat.tref);
        if (mat.has_alpha) d.any_expansion = true;
    }
    if (m.t.empty()) {
        m.t.push_back(0.0);
        m.v.push_back(0.0);
    }
    return d;
}

}  // namespace fx
