// tuner.cpp -- the tuning table (tuner.h).  The measurement itself lives in
// api.cpp (ParODE_TuneResponseBlock), which builds the candidate plans.
#include "tuner.h"

#include "common.h"

#include <map>
#include <mutex>
#include <sstream>
#include <tuple>

namespace parode {

namespace {

using Key = std::tuple<int, int, int, int, int, int>;

struct Entry {
    int log2B = -1;
    float ms = 0.f;
};

std::mutex g_mu;
std::map<Key, Entry>& table()
{
    static std::map<Key, Entry>* t = new std::map<Key, Entry>();
    return *t;
}

Key key_of(const TuneClass& c) { return Key(c.solver, c.np, c.m, c.p, c.tclass, c.precision); }

int pow2_at_least(long v)
{
    int p = 1;
    while (p < v) p <<= 1;
    return p;
}

}  // namespace

TuneClass tune_class(int solver, int Ns, int m, int p, long nScan, int precision)
{
    TuneClass c;
    c.solver = solver;
    c.np = pow2_at_least(std::max(8, Ns));
    c.m = pow2_at_least(std::max(1, m));
    c.p = pow2_at_least(std::max(1, p));
    c.tclass = ilog2(std::max(1L, nScan));
    c.precision = precision;
    return c;
}

int tuned_log2_block(const TuneClass& c)
{
    std::lock_guard<std::mutex> g(g_mu);
    auto it = table().find(key_of(c));
    return it == table().end() ? -1 : it->second.log2B;
}

void tune_store(const TuneClass& c, int log2B, float ms)
{
    std::lock_guard<std::mutex> g(g_mu);
    table()[key_of(c)] = Entry{log2B, ms};
}

void tune_clear()
{
    std::lock_guard<std::mutex> g(g_mu);
    table().clear();
}

std::string tune_dump(const std::string& gpu)
{
    std::lock_guard<std::mutex> g(g_mu);
    std::ostringstream os;
    for (const auto& kv : table()) {
        const Key& k = kv.first;
        os << gpu << ' ' << std::get<0>(k) << ' ' << std::get<1>(k) << ' ' << std::get<2>(k) << ' ' << std::get<3>(k)
           << ' ' << std::get<4>(k) << ' ' << std::get<5>(k) << ' ' << kv.second.log2B << ' ' << kv.second.ms << '\n';
    }
    return os.str();
}

int tune_load_text(const std::string& text, const std::string& gpu)
{
    std::istringstream is(text);
    std::string line;
    int n = 0;
    std::lock_guard<std::mutex> g(g_mu);
    while (std::getline(is, line)) {
        std::istringstream ls(line);
        std::string name;
        TuneClass c;
        int log2B = -1;
        float ms = 0.f;
        if (!(ls >> name >> c.solver >> c.np >> c.m >> c.p >> c.tclass >> c.precision >> log2B >> ms)) continue;
        if (name != gpu || log2B < 2 || log2B > 7) continue;
        table()[key_of(c)] = Entry{log2B, ms};
        ++n;
    }
    return n;
}

}  // namespace parode
