// D_map_define<T> semantics of the drop-in map (no device work).
#include <chrono>
#include <cstdio>
#include <random>
#include <stdexcept>

#include "mt_lbm.hpp"

#define CHECK(c)                                                     \
    do {                                                             \
        if (!(c)) {                                                  \
            std::printf("check failed line %d: %s\n", __LINE__, #c); \
            return 1;                                                \
        }                                                            \
    } while (0)

int main()
{
    mt::D_map_define<double> m;
    CHECK(m.empty());
    CHECK(m.insert(std::make_pair(mt::morton(42), 1.5)).second);
    CHECK(!m.insert(std::make_pair(mt::morton(42), 9.0)).second);  // insert does not overwrite
    CHECK(m.at(mt::morton(42)) == 1.5);
    m.insert(std::make_pair(uint64_t(7), 2.0));
    m[mt::morton(100)] = 3.0;  // operator[] default-inserts
    CHECK(m.size() == 3 && m.count(uint64_t(7)) == 1 && m.count(uint64_t(8)) == 0);
    CHECK(m.find(uint64_t(8)) == m.end());
    bool threw = false;
    try {
        m.at(uint64_t(8));
    } catch (const std::out_of_range &) {
        threw = true;
    }
    CHECK(threw);
    uint64_t prev = 0;
    int n = 0;
    for (auto kv : m) {  // ascending key order
        CHECK(kv.first.to_ullong() >= prev);
        prev = kv.first.to_ullong();
        ++n;
    }
    CHECK(n == 3);
    auto it = m.find(mt::morton(100));
    CHECK(it->second == 3.0 && it->first == mt::morton(100));
    it->second = 4.0;
    CHECK(m.at(uint64_t(100)) == 4.0);
    CHECK(m.erase(uint64_t(7)) == 1 && m.erase(uint64_t(7)) == 0 && m.size() == 2);
    mt::D_map_define<double> o;
    o.insert(m.begin(), m.end());
    CHECK(o.size() == 2 && o.at(uint64_t(42)) == 1.5);
    o.swap(m);
    m.clear();
    CHECK(m.empty() && o.size() == 2);

    // bulk insert = one-by-one insert in sequence order (existing keys and the
    // first occurrence of a repeated key keep their values)
    {
        std::mt19937_64 rng(5);
        mt::D_map_define<int> a, b;
        std::vector<std::pair<uint64_t, int>> seq;
        for (int i = 0; i < 20000; ++i) seq.push_back({rng() % 5000 + (i % 3 ? 0 : (uint64_t(1) << 40)), i});
        for (int i = 0; i < 300; ++i) {
            a.insert(std::make_pair(uint64_t(i * 7), -i));
            b.insert(std::make_pair(uint64_t(i * 7), -i));
        }
        for (auto &kv : seq) a.insert(kv);
        b.insert(seq.begin(), seq.end());
        CHECK(a.size() == b.size());
        CHECK(a.keys() == b.keys() && a.values() == b.values());
        mt::D_map_define<int> c, d;
        c.insert(seq.rbegin(), seq.rend());
        for (auto it = seq.rbegin(); it != seq.rend(); ++it) d.insert(*it);
        CHECK(c.keys() == d.keys() && c.values() == d.values());
    }
    // a reference-sized map (8 M cells, random order) fills in bulk
    {
        const size_t n = size_t(8) << 20;
        std::vector<uint64_t> k(n);
        std::vector<double> v(n);
        std::mt19937_64 rng(11);
        for (size_t i = 0; i < n; ++i) {
            k[i] = rng() >> 4;
            v[i] = (double)i;
        }
        mt::D_map_define<double> big;
        auto t0 = std::chrono::steady_clock::now();
        big.insert_bulk(k, v);
        double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        CHECK(big.size() == n);
        for (size_t i = 1; i < n; ++i) CHECK(big.keys()[i - 1] < big.keys()[i]);
        CHECK(big.at(k[12345]) == 12345.0);
        std::printf("8M-key bulk insert: %.3f s\n", secs);
        CHECK(secs < 6.0);  // a bound for a loaded host; 0.9 s measured alone
    }
    std::printf("dmap ok\n");
    return 0;
}
