// tune_cache.cpp -- the stage-launch autotuner's persistent choices.
//
// One entry per (GPU name, SM count, form, patch size, quad-count bucket):
// the chosen launch shape and its measured time per residual stage. Kept in
// memory for the process and in a JSON file so that later processes on the
// same GPU model skip the timing:
//   AMRGPU_TUNE_CACHE=<path>   the file (empty: memory only)
//   default                    $XDG_CACHE_HOME/amrgpu/tune.json, else
//                              $HOME/.cache/amrgpu/tune.json
// The file is {"amrgpu_tune": 1, "entries": [ {...}, ... ]} with one entry
// object per line; it is rewritten through a temporary file and a rename,
// so a reader never sees a half-written file. Unreadable or malformed
// lines are skipped.
#include <sys/stat.h>
#include <unistd.h>

#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "amrgpu_internal.h"

namespace amrgpu {

namespace {

std::mutex g_mu;
std::vector<TuneEntry> g_entries;
bool g_loaded = false;

bool same_key(const TuneEntry &a, const TuneEntry &b)
{
    return a.gpu == b.gpu && a.sms == b.sms && a.form == b.form && a.n == b.n && a.bucket == b.bucket;
}

void mkdirs(const std::string &dir)
{
    for (size_t p = 1; p <= dir.size(); ++p)
        if (p == dir.size() || dir[p] == '/') mkdir(dir.substr(0, p).c_str(), 0755);
}

void load_locked()
{
    if (g_loaded) return;
    g_loaded = true;
    const std::string path = tune_cache_path();
    if (path.empty()) return;
    FILE *fp = std::fopen(path.c_str(), "r");
    if (!fp) return;
    char line[512];
    while (std::fgets(line, sizeof(line), fp)) {
        const char *p = std::strstr(line, "{\"gpu\": \"");
        if (!p) continue;
        TuneEntry e;
        char name[160] = {0};
        if (std::sscanf(p,
                        "{\"gpu\": \"%159[^\"]\", \"sms\": %d, \"form\": %d, \"n\": %d, \"bucket\": %d, "
                        "\"qpb\": %d, \"threads\": %d, \"min_blocks\": %d, \"ms\": %lf}",
                        name, &e.sms, &e.form, &e.n, &e.bucket, &e.qpb, &e.threads, &e.min_blocks, &e.ms) != 9)
            continue;
        e.gpu = name;
        bool dup = false;
        for (const TuneEntry &o : g_entries) dup |= same_key(o, e);
        if (!dup) g_entries.push_back(e);
    }
    std::fclose(fp);
}

void save_locked()
{
    const std::string path = tune_cache_path();
    if (path.empty()) return;
    const size_t slash = path.rfind('/');
    if (slash != std::string::npos) mkdirs(path.substr(0, slash));
    const std::string tmp = path + ".tmp." + std::to_string((long)getpid());
    FILE *fp = std::fopen(tmp.c_str(), "w");
    if (!fp) return;  // read-only location: the choices stay in memory
    std::fprintf(fp, "{\"amrgpu_tune\": 1, \"entries\": [\n");
    for (size_t k = 0; k < g_entries.size(); ++k) {
        const TuneEntry &e = g_entries[k];
        std::fprintf(fp,
                     "{\"gpu\": \"%s\", \"sms\": %d, \"form\": %d, \"n\": %d, \"bucket\": %d, \"qpb\": %d, "
                     "\"threads\": %d, \"min_blocks\": %d, \"ms\": %.6f}%s\n",
                     e.gpu.c_str(), e.sms, e.form, e.n, e.bucket, e.qpb, e.threads, e.min_blocks, e.ms,
                     k + 1 < g_entries.size() ? "," : "");
    }
    std::fprintf(fp, "]}\n");
    const bool ok = std::fclose(fp) == 0;
    if (!ok || std::rename(tmp.c_str(), path.c_str()) != 0) std::remove(tmp.c_str());
}

}  // namespace

std::string tune_cache_path()
{
    if (const char *p = std::getenv("AMRGPU_TUNE_CACHE")) return std::string(p);
    if (const char *x = std::getenv("XDG_CACHE_HOME"); x && *x) return std::string(x) + "/amrgpu/tune.json";
    if (const char *h = std::getenv("HOME"); h && *h) return std::string(h) + "/.cache/amrgpu/tune.json";
    return std::string();
}

bool tune_lookup(const TuneEntry &key, TuneEntry *out)
{
    std::lock_guard<std::mutex> lk(g_mu);
    load_locked();
    for (const TuneEntry &e : g_entries)
        if (same_key(e, key)) {
            *out = e;
            return true;
        }
    return false;
}

void tune_store(const TuneEntry &e)
{
    std::lock_guard<std::mutex> lk(g_mu);
    load_locked();
    bool found = false;
    for (TuneEntry &o : g_entries)
        if (same_key(o, e)) {
            o = e;
            found = true;
        }
    if (!found) g_entries.push_back(e);
    save_locked();
}

void tune_forget()
{
    std::lock_guard<std::mutex> lk(g_mu);
    g_entries.clear();
    g_loaded = false;
}

}  // namespace amrgpu
