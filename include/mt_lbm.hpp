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
//   Lat_Manager      (header/Lat_Manager.hpp:245-316): the index sets.
//   LBM_Manager      (header/LBM_Manager.hpp:25-119): fluidSimulate,
//       LBMkernel, calculateMacros, AMR_transDDF_explosion/coalescence, and
//       the strategy objects Collision_Model::collide, Stream_Model::stream,
//       ComplexBoundary_Model::treat, D3Q19_BoundaryCondtion_Manager::
//       applyBoundaryCondition.
//
// Failures throw std::runtime_error carrying mt_last_error(); lookups of a
// missing key throw std::out_of_range like the reference's .at().
#pragma once

#include <algorithm>
#include <array>
#include <bitset>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
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
        for (; first != last; ++first) insert(std::make_pair((*first).first, (T)(*first).second));
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

private:
    mt_ctx *h_ = nullptr;
};

class Collision_Model {
public:
    Collision_Model(Context &c, int32_t id) : c_(c), id_(id) {}
    virtual ~Collision_Model() = default;
    virtual void collide(int level) { c_.check(mt_collide(c_.get(), id_, level), "collide"); }
    virtual std::string print_Model_Name() = 0;
protected:
    Context &c_;
    int32_t id_;
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
    Stream_Model(Context &c, int32_t id) : c_(c), id_(id) {}
    virtual ~Stream_Model() = default;
    virtual void stream(int level) = 0;
protected:
    Context &c_;
    int32_t id_;
};
class ABPatternPull : public Stream_Model {
public:
    using Stream_Model::Stream_Model;
    void stream(int level) override { c_.check(mt_stream(c_.get(), id_, level), "stream"); }
};

class ComplexBoundary_Model {
public:
    ComplexBoundary_Model(Context &c, int32_t id) : c_(c), id_(id) {}
    virtual ~ComplexBoundary_Model() = default;
    virtual void treat() = 0;
protected:
    Context &c_;
    int32_t id_;
};
class SinglePointInterpolation : public ComplexBoundary_Model {
public:
    using ComplexBoundary_Model::ComplexBoundary_Model;
    void treat() override { c_.check(mt_ib_treat(c_.get(), id_), "treat"); }
};

class D3Q19_BoundaryCondtion_Manager {
public:
    D3Q19_BoundaryCondtion_Manager(Context &c, int32_t id) : c_(c), id_(id) {}
    void applyBoundaryCondition(const std::string &surface, const std::string &position)
    {
        static const char *names[6] = {"West", "East", "South", "North", "Bot", "Top"};
        if (position != "AfterStream") throw std::invalid_argument("only AfterStream is on the live path");
        for (int f = 0; f < 6; ++f)
            if (surface == names[f]) {
                c_.check(mt_apply_bc_face(c_.get(), id_, f), "applyBoundaryCondition");
                return;
            }
        throw std::invalid_argument("unknown surface " + surface);
    }
private:
    Context &c_;
    int32_t id_;
};

class LBM_Manager {
public:
    LBM_Manager(Context &ctx, Lat_Manager &lat, const mt_case_desc &desc) : ctx_(ctx), desc_(desc)
    {
        ctx_.check(mt_case_create(ctx_.get(), &desc_, &id_), "mt_case_create");
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
        if (desc_.collision == MT_COLL_CUMULANT)
            collideModel.reset(new Collision_Cumulant(ctx_, id_));
        else
            collideModel.reset(new Collision_LBGK(ctx_, id_));
        streamModel.reset(new ABPatternPull(ctx_, id_));
        solidBCModel.reset(new SinglePointInterpolation(ctx_, id_));
        bc_manager_.reset(new D3Q19_BoundaryCondtion_Manager(ctx_, id_));
    }
    ~LBM_Manager() { mt_case_destroy(ctx_.get(), id_); }

    // U_iters coarse steps of LBMkernel(0) + calculateMacros(), graph-replayed
    void fluidSimulate(int iters)
    {
        ctx_.check(mt_step(ctx_.get(), id_, iters), "fluidSimulate");
        ctx_.check(mt_synchronize(ctx_.get()), "synchronize");
    }
    void LBMkernel(int level) { ctx_.check(mt_lbm_kernel(ctx_.get(), id_, level), "LBMkernel"); }
    void calculateMacros(int level) { ctx_.check(mt_calculate_macros(ctx_.get(), id_, level), "calculateMacros"); }
    void calculateMacros()
    {
        for (int l = 0; l <= desc_.max_level; ++l) calculateMacros(l);
    }
    void AMR_transDDF_explosion(int level) { ctx_.check(mt_explosion(ctx_.get(), id_, level), "explosion"); }
    void AMR_transDDF_coalescence(int level) { ctx_.check(mt_coalescence(ctx_.get(), id_, level), "coalescence"); }

    // level data in ascending key order, populations [Q][n]
    std::vector<uint64_t> keys(int level)
    {
        int64_t n = 0;
        ctx_.check(mt_case_level_size(ctx_.get(), id_, level, &n), "level_size");
        std::vector<uint64_t> k((size_t)n);
        ctx_.check(mt_case_get_keys(ctx_.get(), id_, level, k.data(), nullptr), "get_keys");
        return k;
    }
    void populations(int level, std::vector<double> &f, std::vector<double> &fcol)
    {
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
    int32_t id() const { return id_; }

    std::unique_ptr<Collision_Model> collideModel;
    std::unique_ptr<Stream_Model> streamModel;
    std::unique_ptr<ComplexBoundary_Model> solidBCModel;
    std::unique_ptr<D3Q19_BoundaryCondtion_Manager> bc_manager_;

private:
    Context &ctx_;
    mt_case_desc desc_;
    int32_t id_ = -1;
};

}  // namespace mt
