// Online autotuner of launch shapes whose results do not depend on the shape.
//
// A tuned launch (today: the cluster size of the blocked RRQR, whose output is
// bitwise the same for every cluster size) is keyed by a size bucket: device,
// element size, and log2 buckets of the largest rows, the largest columns and
// the number of tasks of the launch. For each key the tuner keeps, per
// candidate, the number of timed launches and the best cost seen (device time
// per unit of algorithmic work, so launches of one bucket with different
// ranks compare fairly).
//
// Modes: 0 = off (the caller's default shape), 1 = online (default: every
// fitting candidate is timed kTries times as launches of its bucket come, then
// the cheapest is used), 2 = frozen (the table only, e.g. one loaded from a
// file; the default where a bucket has no complete entry). The table is
// process-wide and shared by every handle; save/load write and read a plain
// text file of one line per (key, candidate).
#pragma once

#include <map>
#include <mutex>
#include <string>
#include <vector>

namespace spq {

struct TuneKey {
    int kind;  // 0: blocked RRQR cluster size
    int dev, elem, mb, nb, tb;
    bool operator<(const TuneKey& o) const;
};

class Autotuner {
public:
    static constexpr int kTries = 2;
    static Autotuner& get();
    static int bucket(long long v);  // ceil(log2(max(v, 1)))

    int mode() const;
    void set_mode(int mode);
    // The candidate to launch for key: the default in mode 0, the cheapest
    // explored candidate once every one of cands has kTries timings, else (mode
    // 1) the first candidate still short of samples, starting with dflt.
    int choose(const TuneKey& key, const std::vector<int>& cands, int dflt);
    void record(const TuneKey& key, int cand, double cost);
    void reset();
    int entries() const;  // number of (key, candidate) records
    // timed launches still needed before every key seen so far has all its
    // candidates explored (mode 1)
    int pending() const;
    bool save(const std::string& path) const;
    bool load(const std::string& path);

private:
    struct Rec {
        int count = 0;
        double best = 0;
    };
    mutable std::mutex mu_;
    int mode_ = 1;
    std::map<TuneKey, std::map<int, Rec>> tab_;
    std::map<TuneKey, std::vector<int>> cands_;  // candidates offered for each key
};

}  // namespace spq
