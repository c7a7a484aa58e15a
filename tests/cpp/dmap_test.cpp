// D_map_define<T> semantics of the drop-in map (no device work).
#include <cstdio>
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
    std::printf("dmap ok\n");
    return 0;
}
