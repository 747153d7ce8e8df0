#include "autotune.hpp"

#include <algorithm>
#include <cstdio>
#include <tuple>

namespace spq {

bool TuneKey::operator<(const TuneKey& o) const {
    return std::tie(kind, dev, elem, mb, nb, tb) < std::tie(o.kind, o.dev, o.elem, o.mb, o.nb, o.tb);
}

Autotuner& Autotuner::get() {
    static Autotuner t;
    return t;
}

int Autotuner::bucket(long long v) {
    int b = 0;
    while ((1LL << b) < v) ++b;
    return b;
}

int Autotuner::mode() const {
    std::lock_guard<std::mutex> g(mu_);
    return mode_;
}

void Autotuner::set_mode(int mode) {
    std::lock_guard<std::mutex> g(mu_);
    mode_ = mode;
}

int Autotuner::choose(const TuneKey& key, const std::vector<int>& cands, int dflt) {
    std::lock_guard<std::mutex> g(mu_);
    if (mode_ == 0 || cands.empty()) return dflt;
    cands_[key] = cands;
    auto it = tab_.find(key);
    int best = -1;
    double bc = 0;
    bool complete = it != tab_.end();
    for (int c : cands) {
        const Rec* r = nullptr;
        if (it != tab_.end()) {
            auto jt = it->second.find(c);
            if (jt != it->second.end()) r = &jt->second;
        }
        if (!r || r->count < kTries) {
            complete = false;
            continue;
        }
        if (best < 0 || r->best < bc) {
            best = c;
            bc = r->best;
        }
    }
    if (complete) return best;
    if (mode_ == 2) return dflt;
    // explore: the default first, then the other candidates in order
    auto short_of = [&](int c) {
        if (it == tab_.end()) return true;
        auto jt = it->second.find(c);
        return jt == it->second.end() || jt->second.count < kTries;
    };
    for (int c : cands)
        if (c == dflt && short_of(c)) return c;
    for (int c : cands)
        if (short_of(c)) return c;
    return dflt;
}

void Autotuner::record(const TuneKey& key, int cand, double cost) {
    std::lock_guard<std::mutex> g(mu_);
    if (mode_ != 1 || !(cost > 0)) return;
    Rec& r = tab_[key][cand];
    r.best = r.count == 0 ? cost : std::min(r.best, cost);
    r.count += 1;
}

void Autotuner::reset() {
    std::lock_guard<std::mutex> g(mu_);
    tab_.clear();
    cands_.clear();
}

int Autotuner::pending() const {
    std::lock_guard<std::mutex> g(mu_);
    int n = 0;
    for (auto& kv : cands_) {
        auto it = tab_.find(kv.first);
        for (int c : kv.second) {
            int have = 0;
            if (it != tab_.end()) {
                auto jt = it->second.find(c);
                if (jt != it->second.end()) have = jt->second.count;
            }
            n += std::max(0, kTries - have);
        }
    }
    return n;
}

int Autotuner::entries() const {
    std::lock_guard<std::mutex> g(mu_);
    int n = 0;
    for (auto& kv : tab_) n += (int)kv.second.size();
    return n;
}

bool Autotuner::save(const std::string& path) const {
    std::lock_guard<std::mutex> g(mu_);
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) return false;
    std::fprintf(f, "# kind dev elem rows_log2 cols_log2 tasks_log2 candidate count best_cost\n");
    for (auto& kv : tab_)
        for (auto& c : kv.second)
            std::fprintf(f, "%d %d %d %d %d %d %d %d %.9e\n", kv.first.kind, kv.first.dev, kv.first.elem, kv.first.mb,
                         kv.first.nb, kv.first.tb, c.first, c.second.count, c.second.best);
    return std::fclose(f) == 0;
}

bool Autotuner::load(const std::string& path) {
    FILE* f = std::fopen(path.c_str(), "r");
    if (!f) return false;
    std::map<TuneKey, std::map<int, Rec>> tab;
    char line[512];
    bool ok = true;
    while (std::fgets(line, sizeof line, f)) {
        if (line[0] == '#' || line[0] == '\n') continue;
        TuneKey k{};
        int cand = 0;
        Rec r;
        if (std::sscanf(line, "%d %d %d %d %d %d %d %d %lf", &k.kind, &k.dev, &k.elem, &k.mb, &k.nb, &k.tb, &cand,
                        &r.count, &r.best) != 9 ||
            r.count < 0 || cand < 1) {
            ok = false;
            break;
        }
        tab[k][cand] = r;
    }
    std::fclose(f);
    if (!ok) return false;
    std::lock_guard<std::mutex> g(mu_);
    for (auto& kv : tab)
        for (auto& c : kv.second) tab_[kv.first][c.first] = c.second;
    return true;
}

}  // namespace spq
