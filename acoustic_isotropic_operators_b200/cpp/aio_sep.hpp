// Minimal SEP-compatible containers for the reference-facing operator classes.
//
// The reference's host classes take SEP ioLibs types (sep-iolibs, not vendored
// with the reference and not present here): float{1,2,3}DReg regular arrays over
// a hypercube of axes, and paramObj parameter dictionaries. This header gives
// the subset of that interface the operator layer and its callers use — axes
// (n, o, d), getHyper()->getAxis(i) with 1-based i, getVals(), the nested
// accessor (*v->_mat)[i][j], scale / scaleAdd / clone / cloneSpace / random /
// dot / checkSame / min / max, and paramObj getInt / getFloat / getString /
// getInts with and without defaults — with the same meaning, so code written
// against the reference's classes compiles against these unchanged.
//
// Layout: axis 1 is fastest; a float2DReg over (z, x) stores (iz, ix) at
// ix*nz + iz, exactly the slice layout of the C ABI.
#pragma once
#include <cmath>
#include <cstdint>
#include <map>
#include <memory>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace SEP {

struct axis {
    int n = 1;
    float o = 0.f, d = 1.f;
    std::string label, unit;
    axis() = default;
    axis(int n_, float o_ = 0.f, float d_ = 1.f, const std::string& l = "", const std::string& u = "")
        : n(n_), o(o_), d(d_), label(l), unit(u) {}
};

class hypercube {
  public:
    hypercube() = default;
    explicit hypercube(const std::vector<axis>& a) : _axes(a) {}
    hypercube(const axis& a1) : _axes{a1} {}
    hypercube(const axis& a1, const axis& a2) : _axes{a1, a2} {}
    hypercube(const axis& a1, const axis& a2, const axis& a3) : _axes{a1, a2, a3} {}
    // 1-based like the reference (getAxis(1) is the fastest axis); missing axes have n = 1
    axis getAxis(int i) const { return (i >= 1 && i <= (int)_axes.size()) ? _axes[i - 1] : axis(1); }
    std::vector<axis> getAxes() const { return _axes; }
    int getNdim() const { return (int)_axes.size(); }
    void addAxis(const axis& a) { _axes.push_back(a); }
    long long getN123() const {
        long long n = 1;
        for (const auto& a : _axes) n *= a.n;
        return n;
    }
    std::vector<int> getNs() const {
        std::vector<int> ns;
        for (const auto& a : _axes) ns.push_back(a.n);
        return ns;
    }
    bool sameSize(const hypercube& o) const {
        if (getN123() != o.getN123()) return false;
        const int nd = std::max(getNdim(), o.getNdim());
        for (int i = 1; i <= nd; i++)
            if (getAxis(i).n != o.getAxis(i).n) return false;
        return true;
    }

  private:
    std::vector<axis> _axes;
};

// Nested accessors over a contiguous buffer (slowest index first, like the reference's _mat).
struct float1D {
    float* p;
    long long n1;
    float& operator[](long long i) const { return p[i]; }
};
struct float2D {
    float* p;
    long long n1, n2;
    float* operator[](long long i2) const { return p + i2 * n1; }
};
struct float3DRow {
    float* p;
    long long n1;
    float* operator[](long long i2) const { return p + i2 * n1; }
};
struct float3D {
    float* p;
    long long n1, n2, n3;
    float3DRow operator[](long long i3) const { return float3DRow{p + i3 * n1 * n2, n1}; }
};

template <int N, class MAT>
class floatNDReg {
  public:
    using self = floatNDReg<N, MAT>;
    explicit floatNDReg(std::shared_ptr<hypercube> h) : _hyper(std::move(h)) { alloc(); }
    explicit floatNDReg(const hypercube& h) : _hyper(std::make_shared<hypercube>(h)) { alloc(); }

    std::shared_ptr<hypercube> getHyper() const { return _hyper; }
    float* getVals() { return _data.data(); }
    const float* getVals() const { return _data.data(); }
    long long size() const { return (long long)_data.size(); }

    void scale(double s) {
        for (auto& v : _data) v = (float)(v * s);
    }
    void set(float v) { std::fill(_data.begin(), _data.end(), v); }
    void zero() { set(0.f); }
    // this = sc1 * this + sc2 * other
    void scaleAdd(const std::shared_ptr<self> other, double sc1, double sc2) {
        checkSameOrThrow(other);
        const float* o = other->getVals();
        for (size_t i = 0; i < _data.size(); i++) _data[i] = (float)(sc1 * _data[i] + sc2 * o[i]);
    }
    void add(const std::shared_ptr<self> other) { scaleAdd(other, 1.0, 1.0); }
    std::shared_ptr<self> clone() const {
        auto c = std::make_shared<self>(_hyper);
        c->_data = _data;
        return c;
    }
    std::shared_ptr<self> cloneSpace() const { return std::make_shared<self>(_hyper); }
    // uniform in [-1, 1), a fresh stream per call
    void random() {
        static std::mt19937_64 gen(20240601ULL);
        std::uniform_real_distribution<float> u(-1.f, 1.f);
        for (auto& v : _data) v = u(gen);
    }
    double dot(const std::shared_ptr<self> other) const {
        checkSameOrThrow(other);
        const float* o = other->getVals();
        double s = 0.0;
        for (size_t i = 0; i < _data.size(); i++) s += (double)_data[i] * (double)o[i];
        return s;
    }
    bool checkSame(const std::shared_ptr<self> other) const { return other && _hyper->sameSize(*other->getHyper()); }
    float max() const {
        float m = -INFINITY;
        for (float v : _data) m = std::max(m, v);
        return m;
    }
    float min() const {
        float m = INFINITY;
        for (float v : _data) m = std::min(m, v);
        return m;
    }

    std::shared_ptr<MAT> _mat;

  private:
    void alloc() {
        _data.assign((size_t)_hyper->getN123(), 0.f);
        bind();
    }
    void bind();
    void checkSameOrThrow(const std::shared_ptr<self>& o) const {
        if (!checkSame(o)) throw std::runtime_error("SEP vectors of different sizes");
    }
    std::shared_ptr<hypercube> _hyper;
    std::vector<float> _data;
};

template <>
inline void floatNDReg<1, float1D>::bind() {
    _mat = std::make_shared<float1D>(float1D{_data.data(), _hyper->getAxis(1).n});
}
template <>
inline void floatNDReg<2, float2D>::bind() {
    _mat = std::make_shared<float2D>(float2D{_data.data(), _hyper->getAxis(1).n, _hyper->getAxis(2).n});
}
template <>
inline void floatNDReg<3, float3D>::bind() {
    _mat = std::make_shared<float3D>(
        float3D{_data.data(), _hyper->getAxis(1).n, _hyper->getAxis(2).n, _hyper->getAxis(3).n});
}

class float1DReg : public floatNDReg<1, float1D> {
  public:
    using floatNDReg::floatNDReg;
    explicit float1DReg(int n1) : floatNDReg(std::make_shared<hypercube>(axis(n1))) {}
    explicit float1DReg(const axis& a1) : floatNDReg(std::make_shared<hypercube>(a1)) {}
    std::shared_ptr<float1DReg> clone() const { return copyAs<float1DReg>(); }
    std::shared_ptr<float1DReg> cloneSpace() const { return std::make_shared<float1DReg>(getHyper()); }
    double dot(const std::shared_ptr<float1DReg> o) const { return floatNDReg::dot(o); }
    void scaleAdd(const std::shared_ptr<float1DReg> o, double a, double b) { floatNDReg::scaleAdd(o, a, b); }
    bool checkSame(const std::shared_ptr<float1DReg> o) const { return floatNDReg::checkSame(o); }

  private:
    template <class T>
    std::shared_ptr<T> copyAs() const {
        auto c = std::make_shared<T>(getHyper());
        std::copy(getVals(), getVals() + size(), c->getVals());
        return c;
    }
};

class float2DReg : public floatNDReg<2, float2D> {
  public:
    using floatNDReg::floatNDReg;
    float2DReg(int n1, int n2) : floatNDReg(std::make_shared<hypercube>(axis(n1), axis(n2))) {}
    float2DReg(const axis& a1, const axis& a2) : floatNDReg(std::make_shared<hypercube>(a1, a2)) {}
    std::shared_ptr<float2DReg> clone() const {
        auto c = std::make_shared<float2DReg>(getHyper());
        std::copy(getVals(), getVals() + size(), c->getVals());
        return c;
    }
    std::shared_ptr<float2DReg> cloneSpace() const { return std::make_shared<float2DReg>(getHyper()); }
    double dot(const std::shared_ptr<float2DReg> o) const { return floatNDReg::dot(o); }
    void scaleAdd(const std::shared_ptr<float2DReg> o, double a, double b) { floatNDReg::scaleAdd(o, a, b); }
    bool checkSame(const std::shared_ptr<float2DReg> o) const { return floatNDReg::checkSame(o); }
};

class float3DReg : public floatNDReg<3, float3D> {
  public:
    using floatNDReg::floatNDReg;
    float3DReg(int n1, int n2, int n3) : floatNDReg(std::make_shared<hypercube>(axis(n1), axis(n2), axis(n3))) {}
    float3DReg(const axis& a1, const axis& a2, const axis& a3) : floatNDReg(std::make_shared<hypercube>(a1, a2, a3)) {}
    std::shared_ptr<float3DReg> clone() const {
        auto c = std::make_shared<float3DReg>(getHyper());
        std::copy(getVals(), getVals() + size(), c->getVals());
        return c;
    }
    std::shared_ptr<float3DReg> cloneSpace() const { return std::make_shared<float3DReg>(getHyper()); }
    double dot(const std::shared_ptr<float3DReg> o) const { return floatNDReg::dot(o); }
    void scaleAdd(const std::shared_ptr<float3DReg> o, double a, double b) { floatNDReg::scaleAdd(o, a, b); }
    bool checkSame(const std::shared_ptr<float3DReg> o) const { return floatNDReg::checkSame(o); }
};

}  // namespace SEP

// Parameter dictionary (genericIO paramObj): typed getters with and without
// defaults. A missing key without default throws std::runtime_error, as the
// reference's parameter readers abort on it.
class paramObj {
  public:
    virtual ~paramObj() = default;
    virtual bool has(const std::string& k) const = 0;
    virtual std::string raw(const std::string& k) const = 0;

    int getInt(const std::string& k) const { return std::stoi(need(k)); }
    int getInt(const std::string& k, int def) const { return has(k) ? std::stoi(raw(k)) : def; }
    float getFloat(const std::string& k) const { return std::stof(need(k)); }
    float getFloat(const std::string& k, float def) const { return has(k) ? std::stof(raw(k)) : def; }
    std::string getString(const std::string& k) const { return need(k); }
    std::string getString(const std::string& k, const std::string& def) const { return has(k) ? raw(k) : def; }
    std::vector<int> getInts(const std::string& k) const { return parseInts(need(k)); }
    std::vector<int> getInts(const std::string& k, const std::vector<int>& def) const {
        return has(k) ? parseInts(raw(k)) : def;
    }

  private:
    std::string need(const std::string& k) const {
        if (!has(k)) throw std::runtime_error("missing parameter: " + k);
        return raw(k);
    }
    static std::vector<int> parseInts(const std::string& s) {
        std::vector<int> v;
        std::stringstream ss(s);
        std::string tok;
        while (std::getline(ss, tok, ',')) {
            if (!tok.empty()) v.push_back(std::stoi(tok));
        }
        return v;
    }
};

// paramObj over an in-memory key -> value map (values as they would appear in a par file).
class dictParams : public paramObj {
  public:
    dictParams() = default;
    explicit dictParams(const std::map<std::string, std::string>& m) : _m(m) {}
    void set(const std::string& k, const std::string& v) { _m[k] = v; }
    bool has(const std::string& k) const override { return _m.count(k) > 0; }
    std::string raw(const std::string& k) const override { return _m.at(k); }

  private:
    std::map<std::string, std::string> _m;
};
