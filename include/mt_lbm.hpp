// mt_lbm.hpp -- C++17 drop-in layer over the C ABI in mt_lbm.h.
//
// It keeps the names and call shapes a user of MortonTrieCode-CAD2025/
// mortonTrie_AMR already writes against, with the work done by libmtlbm:
//
//   D_map_define<T>  (header/Grid_Class.h:116-137): MortonSoAMap<T>, a
//       Morton-keyed map stored as sorted key / value arrays (insert without
//       overwrite, find, at throwing std::out_of_range, operator[], count,
//       erase, size, empty, clear, swap, emplace, forward iteration with
//       ->first / ->second in ascending key order, as the MortonTrie
//       backend iterates, mortonTrieMap.cpp:18-43).
//       insert(first, last) of n pairs costs O(n + m) after a radix sort of
//       the new keys (m = keys already present), so reference-sized maps
//       can be filled in bulk; a single insert is O(m).
//   Lat_Manager      (header/Lat_Manager.hpp:245-316): the index sets, and
//       the Lat_Manager::pointer_me singleton (Lat_Manager.hpp:242).
//   LBM_Manager      (header/LBM_Manager.hpp:25-119): fluidSimulate,
//       LBMkernel, calculateMacros, AMR_transDDF_explosion/coalescence, and
//       the strategy objects Collision_Model::collide, Stream_Model::stream,
//       ComplexBoundary_Model::treat, D3Q19_BoundaryCondtion_Manager::
//       applyBoundaryCondition; LBM_Manager::pointer_me and the
//       no-argument constructor (LBM_Manager.hpp:113-115), which reads the
//       index sets from Lat_Manager::pointer_me and the case constants from
//       LBM_Manager::config(), as the reference reads its Constants.h.
//   User[level]      (header/user.h:18-45,154-167): user[l].df.f[q].at(code),
//       df.fcol[q].at(code), density.at(code), velocity.at(code) by Morton
//       code, over a host copy of the level that is read back in bulk on the
//       first access after device work and written back in bulk (when a
//       population was changed) before the next device call.
//
// Failures throw std::runtime_error carrying mt_last_error(); lookups of a
// missing key throw std::out_of_range like the reference's .at().
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <bitset>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "mt_lbm.h"

namespace mt {

using morton = std::bitset<64>;
inline uint64_t key_of(const morton &k) { return k.to_ullong(); }
inline uint64_t key_of(uint64_t k) { return k; }

template <class T> class MortonSoAMap {
public:
    struct proxy {
        morton first;
        T &second;
        proxy *operator->() { return this; }
    };
    class iterator {
    public:
        iterator(MortonSoAMap *m, size_t i) : m_(m), i_(i) {}
        proxy operator*() const { return proxy{morton(m_->keys_[i_]), m_->vals_[i_]}; }
        proxy operator->() const { return **this; }
        iterator &operator++() { ++i_; return *this; }
        bool operator==(const iterator &o) const { return i_ == o.i_ && m_ == o.m_; }
        bool operator!=(const iterator &o) const { return !(*this == o); }
        size_t index() const { return i_; }
    private:
        MortonSoAMap *m_;
        size_t i_;
    };

    template <class K> std::pair<iterator, bool> insert(const std::pair<K, T> &kv)
    {
        const uint64_t k = key_of(kv.first);
        size_t i = lower(k);
        if (i < keys_.size() && keys_[i] == k) return {iterator(this, i), false};
        keys_.insert(keys_.begin() + (std::ptrdiff_t)i, k);
        vals_.insert(vals_.begin() + (std::ptrdiff_t)i, kv.second);
        return {iterator(this, i), true};
    }
    template <class It> void insert(It first, It last)
    {
        std::vector<uint64_t> nk;
        std::vector<T> nv;
        for (; first != last; ++first) {
            nk.push_back(key_of((*first).first));
            nv.push_back((T)(*first).second);
        }
        insert_bulk(nk, nv);
    }
    // the pairs (nk[i], nv[i]) in any order, with the result of inserting
    // them one by one in that order: a key already in the map, or met earlier
    // in the sequence, keeps its value.  Stable LSD radix sort of the new keys
    // (11-bit digits, digits equal across all keys skipped), then one merge.
    void insert_bulk(const std::vector<uint64_t> &nk, const std::vector<T> &nv)
    {
        const size_t m = nk.size();
        if (nv.size() != m) throw std::invalid_argument("insert_bulk: key and value counts differ");
        if (m > 0xFFFFFFFFull) throw std::length_error("insert_bulk: more than 2^32 pairs in one call");
        if (!m) return;
        // keys travel with their sequence positions, so each pass reads both
        // arrays in order; 11-bit digits keep the 2048 scatter targets in cache
        std::vector<uint64_t> kk(nk), kt(m);
        std::vector<uint32_t> ord(m), tmp(m);
        for (size_t i = 0; i < m; ++i) ord[i] = (uint32_t)i;
        uint64_t all_or = 0, all_and = ~uint64_t(0);
        for (uint64_t k : nk) {
            all_or |= k;
            all_and &= k;
        }
        constexpr int kBits = 11;
        constexpr uint64_t kMask = (uint64_t(1) << kBits) - 1;
        std::vector<size_t> cnt(kMask + 2);
        for (int sh = 0; sh < 64; sh += kBits) {
            if ((((all_or ^ all_and) >> sh) & kMask) == 0) continue;  // same digit everywhere
            std::fill(cnt.begin(), cnt.end(), 0);
            for (size_t i = 0; i < m; ++i) ++cnt[((kk[i] >> sh) & kMask) + 1];
            for (size_t b = 1; b < cnt.size(); ++b) cnt[b] += cnt[b - 1];
            for (size_t i = 0; i < m; ++i) {
                const size_t dst = cnt[(kk[i] >> sh) & kMask]++;
                kt[dst] = kk[i];
                tmp[dst] = ord[i];
            }
            kk.swap(kt);
            ord.swap(tmp);
        }
        std::vector<uint64_t> k2;
        std::vector<T> v2;
        k2.reserve(keys_.size() + m);
        v2.reserve(keys_.size() + m);
        size_t a = 0, j = 0;
        while (a < keys_.size() || j < m) {
            if (j < m && j > 0 && kk[j] == kk[j - 1]) {  // later duplicate in the sequence
                ++j;
                continue;
            }
            if (j >= m || (a < keys_.size() && keys_[a] <= kk[j])) {
                if (j < m && keys_[a] == kk[j]) ++j;  // present already: keeps its value
                k2.push_back(keys_[a]);
                v2.push_back(std::move(vals_[a]));
                ++a;
            } else {
                k2.push_back(kk[j]);
                v2.push_back(nv[ord[j]]);
                ++j;
            }
        }
        keys_.swap(k2);
        vals_.swap(v2);
    }
    void reserve(size_t n)
    {
        keys_.reserve(n);
        vals_.reserve(n);
    }
    template <class K, class... A> std::pair<iterator, bool> emplace(const K &k, A &&...a)
    {
        return insert(std::make_pair(k, T(std::forward<A>(a)...)));
    }
    template <class K> iterator find(const K &key)
    {
        const uint64_t k = key_of(key);
        size_t i = lower(k);
        return (i < keys_.size() && keys_[i] == k) ? iterator(this, i) : end();
    }
    template <class K> T &at(const K &key)
    {
        iterator it = find(key);
        if (it == end()) throw std::out_of_range("MortonSoAMap::at: key not present");
        return vals_[it.index()];
    }
    template <class K> T &operator[](const K &key) { return vals_[insert(std::make_pair(key_of(key), T())).first.index()]; }
    template <class K> size_t count(const K &key) { return find(key) == end() ? 0 : 1; }
    template <class K> size_t erase(const K &key)
    {
        iterator it = find(key);
        if (it == end()) return 0;
        keys_.erase(keys_.begin() + (std::ptrdiff_t)it.index());
        vals_.erase(vals_.begin() + (std::ptrdiff_t)it.index());
        return 1;
    }
    size_t size() const { return keys_.size(); }
    bool empty() const { return keys_.empty(); }
    void clear() { keys_.clear(); vals_.clear(); }
    void swap(MortonSoAMap &o) { keys_.swap(o.keys_); vals_.swap(o.vals_); }
    iterator begin() { return iterator(this, 0); }
    iterator end() { return iterator(this, keys_.size()); }
    const std::vector<uint64_t> &keys() const { return keys_; }
    const std::vector<T> &values() const { return vals_; }

private:
    size_t lower(uint64_t k) const { return (size_t)(std::lower_bound(keys_.begin(), keys_.end(), k) - keys_.begin()); }
    std::vector<uint64_t> keys_;
    std::vector<T> vals_;
};

template <class T> using D_map_define = MortonSoAMap<T>;

struct Cell {
    int flag = 0;
};
using D_mapLat = MortonSoAMap<Cell>;

struct Lat_Manager {
    // the most recently constructed Lat_Manager (Lat_Manager.hpp:242)
    inline static Lat_Manager *pointer_me = nullptr;
    Lat_Manager() { pointer_me = this; }
    ~Lat_Manager()
    {
        if (pointer_me == this) pointer_me = nullptr;
    }
    std::array<D_mapLat, MT_MAX_LEVELS> lat_f, lat_overlap_F2C, lat_overlap_C2F, ghost_overlap_C2F,
        ghost_overlap_F2C;
    D_mapLat lat_sf;
    std::array<std::vector<uint64_t>, 26> lat_bc;  // D_setLat per boundary set
    MortonSoAMap<std::vector<double>> dis;         // Q-1 wall distances per IB cell
};

class Context {
public:
    explicit Context(int device = 0)
    {
        if (mt_create(device, &h_) != MT_OK) throw std::runtime_error("mt_create failed");
    }
    ~Context() { if (h_) mt_destroy(h_); }
    Context(const Context &) = delete;
    Context &operator=(const Context &) = delete;
    mt_ctx *get() const { return h_; }
    void check(int rc, const char *what) const
    {
        if (rc != MT_OK) throw std::runtime_error(std::string(what) + ": " + mt_last_error(h_));
    }
    // the process-wide context on device 0 that the no-argument LBM_Manager
    // uses (created on first use, destroyed at exit)
    static Context &shared()
    {
        static Context c(0);
        return c;
    }

private:
    mt_ctx *h_ = nullptr;
};

struct D_uvw {
    double x = 0, y = 0, z = 0;
};

// Host copy of one level of a case: keys, f / fcol [Q][n], density [n],
// velocity [n].  Populations and macros are read back in bulk on the first
// access after device work; a population returned by reference is assumed
// changed, and the level is written back in bulk before the next device call.
class LevelState {
public:
    LevelState(Context &c, int32_t id, int level, int q) : c_(c), id_(id), level_(level), q_(q) {}
    int64_t index(uint64_t k)
    {
        load_keys();
        auto it = std::lower_bound(keys_.begin(), keys_.end(), k);
        return (it != keys_.end() && *it == k) ? (int64_t)(it - keys_.begin()) : -1;
    }
    int64_t at_index(uint64_t k)
    {
        const int64_t i = index(k);
        if (i < 0) throw std::out_of_range("key not stored on this level");
        return i;
    }
    double &pop(bool col, int q, uint64_t k)
    {
        if (q < 0 || q >= q_) throw std::out_of_range("direction out of range");
        const int64_t i = at_index(k);
        load_pops();
        dirty_ = true;
        return (col ? fcol_ : f_)[(size_t)q * keys_.size() + (size_t)i];
    }
    const double &density(uint64_t k)
    {
        const int64_t i = at_index(k);
        load_macros();
        return rho_[(size_t)i];
    }
    const D_uvw &velocity(uint64_t k)
    {
        const int64_t i = at_index(k);
        load_macros();
        return vel_[(size_t)i];
    }
    const std::vector<uint64_t> &keys()
    {
        load_keys();
        return keys_;
    }
    // before a device call: changed populations go back to the device
    void flush()
    {
        if (!dirty_) return;
        c_.check(mt_case_set_populations(c_.get(), id_, level_, f_.data(), fcol_.data()), "set_populations");
        dirty_ = false;
    }
    // after a device call: the host copies are stale
    void invalidate()
    {
        pops_ = macros_ = false;
    }

private:
    void load_keys()
    {
        if (keys_loaded_) return;
        int64_t n = 0;
        c_.check(mt_case_level_size(c_.get(), id_, level_, &n), "level_size");
        keys_.resize((size_t)n);
        if (n) c_.check(mt_case_get_keys(c_.get(), id_, level_, keys_.data(), nullptr), "get_keys");
        keys_loaded_ = true;
    }
    void load_pops()
    {
        if (pops_) return;
        load_keys();
        f_.resize(keys_.size() * (size_t)q_);
        fcol_.resize(keys_.size() * (size_t)q_);
        if (!keys_.empty())
            c_.check(mt_case_get_populations(c_.get(), id_, level_, f_.data(), fcol_.data()), "get_populations");
        pops_ = true;
    }
    void load_macros()
    {
        if (macros_) return;
        flush();
        load_keys();
        const size_t n = keys_.size();
        rho_.resize(n);
        std::vector<double> u(3 * n);
        if (n) c_.check(mt_case_get_macros(c_.get(), id_, level_, rho_.data(), u.data()), "get_macros");
        vel_.resize(n);
        for (size_t i = 0; i < n; ++i) vel_[i] = D_uvw{u[i], u[n + i], u[2 * n + i]};
        macros_ = true;
    }
    Context &c_;
    int32_t id_;
    int level_, q_;
    bool keys_loaded_ = false, pops_ = false, macros_ = false, dirty_ = false;
    std::vector<uint64_t> keys_;
    std::vector<double> f_, fcol_, rho_;
    std::vector<D_uvw> vel_;
};

// One direction of f or fcol of a level by Morton code (user.h:34-45): the
// lattice is fixed, so operator[] finds like at() and inserts nothing.
class DDFSlot {
public:
    void bind(LevelState *s, bool col, int q)
    {
        s_ = s;
        col_ = col;
        q_ = q;
    }
    template <class K> double &at(const K &key) { return s_->pop(col_, q_, key_of(key)); }
    template <class K> double &operator[](const K &key) { return at(key); }
    template <class K> size_t count(const K &key) const { return s_->index(key_of(key)) >= 0 ? 1 : 0; }
    template <class K> bool exists(const K &key) const { return count(key) == 1; }

private:
    LevelState *s_ = nullptr;
    bool col_ = false;
    int q_ = 0;
};

struct _s_DDF {
    DDFSlot f[27];
    DDFSlot fcol[27];
};

// density / velocity maps of a level, read-only (calculateMacros writes them)
template <class V> class MacroView {
public:
    explicit MacroView(LevelState *s = nullptr) : s_(s) {}
    template <class K> const V &at(const K &key) const
    {
        if constexpr (std::is_same<V, D_uvw>::value)
            return s_->velocity(key_of(key));
        else
            return s_->density(key_of(key));
    }
    template <class K> size_t count(const K &key) const { return s_->index(key_of(key)) >= 0 ? 1 : 0; }
    size_t size() const { return s_->keys().size(); }

private:
    LevelState *s_;
};

// User[level] of the reference (user.h:154-167) as views of the device state
struct User {
    _s_DDF df;
    MacroView<double> density;
    MacroView<D_uvw> velocity;
};

// the per-level host copies of one case, shared by the manager and its
// strategy objects: every device call flushes before and invalidates after
class CaseState {
public:
    CaseState(Context &c, int32_t id, int levels, int q) : ctx(c), id(id)
    {
        for (int l = 0; l < levels; ++l) lv.emplace_back(new LevelState(c, id, l, q));
    }
    template <class F> void call(F &&fn)
    {
        for (auto &s : lv) s->flush();
        fn();
        for (auto &s : lv) s->invalidate();
    }
    Context &ctx;
    int32_t id;
    std::vector<std::unique_ptr<LevelState>> lv;
};

class Collision_Model {
public:
    explicit Collision_Model(CaseState &s) : s_(s) {}
    virtual ~Collision_Model() = default;
    virtual void collide(int level)
    {
        s_.call([&] { s_.ctx.check(mt_collide(s_.ctx.get(), s_.id, level), "collide"); });
    }
    virtual std::string print_Model_Name() = 0;
protected:
    CaseState &s_;
};
class Collision_LBGK : public Collision_Model {
public:
    using Collision_Model::Collision_Model;
    std::string print_Model_Name() override { return "LBGK"; }
};
class Collision_Cumulant : public Collision_Model {
public:
    using Collision_Model::Collision_Model;
    std::string print_Model_Name() override { return "Cumulant"; }
};

class Stream_Model {
public:
    explicit Stream_Model(CaseState &s) : s_(s) {}
    virtual ~Stream_Model() = default;
    virtual void stream(int level) = 0;
protected:
    CaseState &s_;
};
class ABPatternPull : public Stream_Model {
public:
    using Stream_Model::Stream_Model;
    void stream(int level) override
    {
        s_.call([&] { s_.ctx.check(mt_stream(s_.ctx.get(), s_.id, level), "stream"); });
    }
};

class ComplexBoundary_Model {
public:
    explicit ComplexBoundary_Model(CaseState &s) : s_(s) {}
    virtual ~ComplexBoundary_Model() = default;
    virtual void treat() = 0;
protected:
    CaseState &s_;
};
class SinglePointInterpolation : public ComplexBoundary_Model {
public:
    using ComplexBoundary_Model::ComplexBoundary_Model;
    void treat() override
    {
        s_.call([&] { s_.ctx.check(mt_ib_treat(s_.ctx.get(), s_.id), "treat"); });
    }
};

class D3Q19_BoundaryCondtion_Manager {
public:
    explicit D3Q19_BoundaryCondtion_Manager(CaseState &s) : s_(s) {}
    void applyBoundaryCondition(const std::string &surface, const std::string &position)
    {
        static const char *names[6] = {"West", "East", "South", "North", "Bot", "Top"};
        if (position != "AfterStream") throw std::invalid_argument("only AfterStream is on the live path");
        for (int f = 0; f < 6; ++f)
            if (surface == names[f]) {
                s_.call([&] { s_.ctx.check(mt_apply_bc_face(s_.ctx.get(), s_.id, f), "applyBoundaryCondition"); });
                return;
            }
        throw std::invalid_argument("unknown surface " + surface);
    }
private:
    CaseState &s_;
};

class LBM_Manager {
public:
    // the most recently constructed manager (LBM_Manager.hpp:115)
    inline static LBM_Manager *pointer_me = nullptr;
    // the case constants the no-argument constructor uses, filled by the
    // caller as the reference's Constants.h fixes them at compile time
    // (lattice, levels, collision, IB method, boundary, tau per level, rho0,
    // boundary velocity, periodic axes and level-0 extent)
    static mt_case_desc &config()
    {
        static mt_case_desc d{};
        return d;
    }

    // LBM_Manager() (LBM_Manager.cpp:32-95): the index sets of
    // Lat_Manager::pointer_me, the constants of config(), the shared context
    LBM_Manager() : LBM_Manager(Context::shared(), lat_or_throw(), config()) {}

    LBM_Manager(Context &ctx, Lat_Manager &lat, const mt_case_desc &desc) : ctx_(ctx), desc_(desc)
    {
        ctx_.check(mt_case_create(ctx_.get(), &desc_, &id_), "mt_case_create");
        try {
            upload(lat);
        } catch (...) {
            mt_case_destroy(ctx_.get(), id_);
            throw;
        }
        state_.reset(new CaseState(ctx_, id_, desc_.max_level + 1, desc_.q));
        users_.resize((size_t)desc_.max_level + 1);
        for (int l = 0; l <= desc_.max_level; ++l) {
            LevelState *s = state_->lv[(size_t)l].get();
            for (int q = 0; q < desc_.q; ++q) {
                users_[(size_t)l].df.f[q].bind(s, false, q);
                users_[(size_t)l].df.fcol[q].bind(s, true, q);
            }
            users_[(size_t)l].density = MacroView<double>(s);
            users_[(size_t)l].velocity = MacroView<D_uvw>(s);
        }
        user = users_.data();
        if (desc_.collision == MT_COLL_CUMULANT)
            collideModel.reset(new Collision_Cumulant(*state_));
        else
            collideModel.reset(new Collision_LBGK(*state_));
        streamModel.reset(new ABPatternPull(*state_));
        solidBCModel.reset(new SinglePointInterpolation(*state_));
        bc_manager_.reset(new D3Q19_BoundaryCondtion_Manager(*state_));
        pointer_me = this;
    }
    ~LBM_Manager()
    {
        if (pointer_me == this) pointer_me = nullptr;
        mt_case_destroy(ctx_.get(), id_);
    }
    LBM_Manager(const LBM_Manager &) = delete;
    LBM_Manager &operator=(const LBM_Manager &) = delete;

    // U_iters coarse steps of LBMkernel(0) + calculateMacros(), graph-replayed
    void fluidSimulate(int iters)
    {
        device([&] {
            ctx_.check(mt_step(ctx_.get(), id_, iters), "fluidSimulate");
            ctx_.check(mt_synchronize(ctx_.get()), "synchronize");
        });
    }
    void LBMkernel(int level)
    {
        device([&] { ctx_.check(mt_lbm_kernel(ctx_.get(), id_, level), "LBMkernel"); });
    }
    void calculateMacros(int level)
    {
        device([&] { ctx_.check(mt_calculate_macros(ctx_.get(), id_, level), "calculateMacros"); });
    }
    void calculateMacros()
    {
        for (int l = 0; l <= desc_.max_level; ++l) calculateMacros(l);
    }
    void AMR_transDDF_explosion(int level)
    {
        device([&] { ctx_.check(mt_explosion(ctx_.get(), id_, level), "explosion"); });
    }
    void AMR_transDDF_coalescence(int level)
    {
        device([&] { ctx_.check(mt_coalescence(ctx_.get(), id_, level), "coalescence"); });
    }

    // level data in ascending key order, populations [Q][n]
    std::vector<uint64_t> keys(int level) { return state_->lv[(size_t)level]->keys(); }
    void populations(int level, std::vector<double> &f, std::vector<double> &fcol)
    {
        device([] {});
        int64_t n = 0;
        ctx_.check(mt_case_level_size(ctx_.get(), id_, level, &n), "level_size");
        f.resize((size_t)(n * desc_.q));
        fcol.resize((size_t)(n * desc_.q));
        ctx_.check(mt_case_get_populations(ctx_.get(), id_, level, f.data(), fcol.data()), "get_populations");
    }
    std::array<double, 4> force()
    {
        std::array<double, 4> out{};
        ctx_.check(mt_get_force(ctx_.get(), id_, out.data()), "get_force");
        return out;
    }
    // A checkpoint of the state between coarse steps (no reference
    // counterpart), one binary file: a header (Q, levels, storage, coarse
    // steps), per level n, its sorted keys and FP64 f and fcol [Q][n], and
    // for direct forcing the band's force field [3][n of the finest level].
    // loadCheckpoint restores it into a case of the same lattice and storage
    // (std::runtime_error otherwise); stepping on then gives what stepping
    // on from the saved case gives.
    // coarse steps taken (mt_case_get_step)
    int64_t coarseSteps()
    {
        int64_t st = 0;
        ctx_.check(mt_case_get_step(ctx_.get(), id_, &st), "get_step");
        return st;
    }
    void saveCheckpoint(const std::string &path)
    {
        device([&] {
            std::FILE *fp = std::fopen(path.c_str(), "wb");
            if (!fp) throw std::runtime_error("saveCheckpoint: cannot open " + path);
            int64_t steps = 0;
            ctx_.check(mt_case_get_step(ctx_.get(), id_, &steps), "get_step");
            const int64_t head[5] = {0x4d54434b50540001LL, desc_.q, desc_.max_level, desc_.storage, steps};
            bool ok = std::fwrite(head, sizeof(head), 1, fp) == 1;
            int64_t nfine = 0;
            for (int l = 0; l <= desc_.max_level && ok; ++l) {
                int64_t n = 0;
                ctx_.check(mt_case_level_size(ctx_.get(), id_, l, &n), "level_size");
                std::vector<uint64_t> k((size_t)n);
                std::vector<uint32_t> tags((size_t)n);
                std::vector<double> f((size_t)(n * desc_.q)), fc((size_t)(n * desc_.q));
                ctx_.check(mt_case_get_keys(ctx_.get(), id_, l, k.data(), tags.data()), "get_keys");
                ctx_.check(mt_case_get_populations(ctx_.get(), id_, l, f.data(), fc.data()), "get_populations");
                ok = std::fwrite(&n, sizeof(n), 1, fp) == 1 && (!n || (std::fwrite(k.data(), 8, k.size(), fp) == k.size() &&
                     std::fwrite(f.data(), 8, f.size(), fp) == f.size() && std::fwrite(fc.data(), 8, fc.size(), fp) == fc.size()));
                nfine = n;
            }
            const int64_t has_df = desc_.ib_method == MT_IB_DF ? 1 : 0;
            ok = ok && std::fwrite(&has_df, sizeof(has_df), 1, fp) == 1;
            if (ok && has_df) {
                std::vector<int64_t> acc((size_t)(3 * nfine));
                ctx_.check(mt_case_get_df_force_field(ctx_.get(), id_, acc.data()), "get_df_force_field");
                ok = std::fwrite(acc.data(), 8, acc.size(), fp) == acc.size();
            }
            if (std::fclose(fp) != 0 || !ok) throw std::runtime_error("saveCheckpoint: write failed: " + path);
        });
    }
    void loadCheckpoint(const std::string &path)
    {
        device([&] {
            std::FILE *fp = std::fopen(path.c_str(), "rb");
            if (!fp) throw std::runtime_error("loadCheckpoint: cannot open " + path);
            auto fail = [&](const std::string &why) {
                std::fclose(fp);
                throw std::runtime_error("loadCheckpoint: " + why);
            };
            int64_t head[5];
            if (std::fread(head, sizeof(head), 1, fp) != 1 || head[0] != 0x4d54434b50540001LL) fail("not a checkpoint");
            if (head[1] != desc_.q || head[2] != desc_.max_level || head[3] != desc_.storage)
                fail("checkpoint of another model, level count or storage");
            std::vector<std::vector<double>> f(desc_.max_level + 1), fc(desc_.max_level + 1);
            int64_t nfine = 0;
            for (int l = 0; l <= desc_.max_level; ++l) {
                int64_t n = 0, m = 0;
                ctx_.check(mt_case_level_size(ctx_.get(), id_, l, &m), "level_size");
                if (std::fread(&n, sizeof(n), 1, fp) != 1 || n != m) fail("checkpoint of another lattice");
                std::vector<uint64_t> k((size_t)n), mine((size_t)n);
                std::vector<uint32_t> tags((size_t)n);
                f[l].resize((size_t)(n * desc_.q));
                fc[l].resize((size_t)(n * desc_.q));
                if (n && (std::fread(k.data(), 8, k.size(), fp) != k.size() ||
                          std::fread(f[l].data(), 8, f[l].size(), fp) != f[l].size() ||
                          std::fread(fc[l].data(), 8, fc[l].size(), fp) != fc[l].size()))
                    fail("truncated file");
                ctx_.check(mt_case_get_keys(ctx_.get(), id_, l, mine.data(), tags.data()), "get_keys");
                if (k != mine) fail("checkpoint of another lattice");
                nfine = n;
            }
            int64_t has_df = 0;
            if (std::fread(&has_df, sizeof(has_df), 1, fp) != 1) fail("truncated file");
            std::vector<int64_t> acc;
            if (has_df) {
                acc.resize((size_t)(3 * nfine));
                if (std::fread(acc.data(), 8, acc.size(), fp) != acc.size()) fail("truncated file");
            }
            std::fclose(fp);
            for (int l = 0; l <= desc_.max_level; ++l)
                ctx_.check(mt_case_set_populations(ctx_.get(), id_, l, f[l].data(), fc[l].data()), "set_populations");
            if (has_df) ctx_.check(mt_case_set_df_force_field(ctx_.get(), id_, acc.data()), "set_df_force_field");
            ctx_.check(mt_case_set_step(ctx_.get(), id_, head[4]), "set_step");
        });
    }
    // FP64 device sums per level and volume-weighted: [(max_level + 2) * 5]
    std::vector<double> reduce_levels()
    {
        std::vector<double> out(5 * (size_t)(desc_.max_level + 2));
        device([&] { ctx_.check(mt_case_reduce_levels(ctx_.get(), id_, out.data()), "reduce_levels"); });
        return out;
    }
    // infoPrint's diagnostics per level: [(max_level + 1) * 4] = max |u|,
    // cells with |u| > 1, sum |u - u_prev|^2, sum |u|^2 (mt_case_info)
    std::vector<double> info()
    {
        std::vector<double> out(4 * (size_t)(desc_.max_level + 1));
        device([&] { ctx_.check(mt_case_info(ctx_.get(), id_, out.data()), "info"); });
        return out;
    }
    // LBM_Manager::infoPrint (LBM_Manager.cpp:914-979): the velocity change
    // since the previous call, per level max |u| / cells above 1, and with a
    // drag scale (u_lb = the boundary velocity in level-0 lattice units,
    // d_lb = the body's diameter in finest cells, both > 0) Cd of the mean
    // force per treat() call since the previous call, whose sums are then
    // reset as the reference resets them
    void infoPrint(long iter_no, double u_lb = 0.0, double d_lb = 0.0, std::FILE *out = stdout)
    {
        const std::vector<double> d = info();
        double e2 = 0.0, v2 = 0.0;
        for (int l = 0; l <= desc_.max_level; ++l) {
            e2 += d[4 * l + 2];
            v2 += d[4 * l + 3];
        }
        std::fprintf(out, "[Iter] %ld Velocity error = %g | max|v|/nbig:", iter_no, std::sqrt(e2) / std::sqrt(v2 + 1e-16));
        for (int l = 0; l <= desc_.max_level; ++l) std::fprintf(out, " L%d=%g/%ld", l, d[4 * l], (long)d[4 * l + 1]);
        const std::array<double, 4> f = force();
        if (u_lb > 0.0 && d_lb > 0.0 && f[3] > 0.0) {
            const double fx = f[0] / f[3];
            const double cd = 2.0 * fx / (u_lb * u_lb * 3.14159265358979323846 * d_lb * d_lb / 4.0);
            cd_sum_ += cd;
            ++cd_count_;
            std::fprintf(out, "  Cd = %g  (Cd_avg = %g, Fx_lb = %g, n = %ld)", cd, cd_sum_ / cd_count_, fx, (long)f[3]);
            ctx_.check(mt_reset_force(ctx_.get(), id_), "reset_force");
        }
        std::fprintf(out, "\n");
    }
    int32_t id() const { return id_; }
    const mt_case_desc &desc() const { return desc_; }

    std::unique_ptr<Collision_Model> collideModel;
    std::unique_ptr<Stream_Model> streamModel;
    std::unique_ptr<ComplexBoundary_Model> solidBCModel;
    std::unique_ptr<D3Q19_BoundaryCondtion_Manager> bc_manager_;
    // user[level] (LBM_Manager.hpp:45): per-key views of the device state
    User *user = nullptr;

private:
    double cd_sum_ = 0.0;
    long cd_count_ = 0;
    static Lat_Manager &lat_or_throw()
    {
        if (!Lat_Manager::pointer_me) throw std::runtime_error("LBM_Manager(): no Lat_Manager constructed");
        return *Lat_Manager::pointer_me;
    }
    template <class F> void device(F &&fn) { state_->call(fn); }
    void upload(Lat_Manager &lat)
    {
        const int L = desc_.max_level;
        auto add = [&](int level, int set, const std::vector<uint64_t> &k) {
            ctx_.check(mt_case_add_set(ctx_.get(), id_, level, set, k.data(), (int64_t)k.size()), "mt_case_add_set");
        };
        for (int l = 0; l <= L; ++l) {
            add(l, MT_SET_LAT_F, lat.lat_f[l].keys());
            add(l, MT_SET_OVERLAP_F2C, lat.lat_overlap_F2C[l].keys());
            add(l, MT_SET_OVERLAP_C2F, lat.lat_overlap_C2F[l].keys());
            add(l, MT_SET_GHOST_C2F, lat.ghost_overlap_C2F[l].keys());
            add(l, MT_SET_GHOST_F2C, lat.ghost_overlap_F2C[l].keys());
        }
        add(L, MT_SET_LAT_SF, lat.lat_sf.keys());
        for (int b = 0; b < 26; ++b) add(0, MT_SET_LAT_BC0 + b, lat.lat_bc[b]);
        std::vector<double> rows;
        for (const auto &r : lat.dis.values()) rows.insert(rows.end(), r.begin(), r.end());
        ctx_.check(mt_case_set_dis(ctx_.get(), id_, lat.dis.keys().data(), rows.data(), (int64_t)lat.dis.size()),
                   "mt_case_set_dis");
        ctx_.check(mt_case_build(ctx_.get(), id_), "mt_case_build");
    }

    Context &ctx_;
    mt_case_desc desc_;
    int32_t id_ = -1;
    std::unique_ptr<CaseState> state_;
    std::vector<User> users_;
};

}  // namespace mt
