// Linear operator interface of the reference (F/include/operator.h:7-100):
// forward(add, model, data) / adjoint(add, model, data), where add = false
// overwrites the output and add = true accumulates into it; a domain / range
// pair set by setDomainRange; and the dot-product test.
#pragma once
#include <cmath>
#include <iomanip>
#include <iostream>
#include <memory>
#include <stdexcept>
#include <string>

#include "aio_b200.h"

template <class V1, class V2>
class Operator {
  public:
    virtual ~Operator() = default;
    virtual void forward(const bool add, const std::shared_ptr<V1> model, std::shared_ptr<V2> data) const = 0;
    virtual void adjoint(const bool add, std::shared_ptr<V1> model, const std::shared_ptr<V2> data) const = 0;

    bool checkDomainRange(const std::shared_ptr<V1> model, const std::shared_ptr<V2> data) const {
        bool ok = true;
        if (!_domain->checkSame(model)) {
            std::cerr << "Domains do not match" << std::endl;
            ok = false;
        }
        if (!_range->checkSame(data)) {
            std::cerr << "Ranges do not match" << std::endl;
            ok = false;
        }
        return ok;
    }

    // <F m, d> against <m, F* d> for random m and d, without and with add; relative
    // error of each pair must not exceed maxError. The inner products accumulate in FP64: for the
    // GPU operators (dotTestDevice() >= 0) exact FP64 products reduced on that GPU in a fixed
    // order (aio_dot_f64), for host operators on the host.
    bool dotTest(const bool verbose = false, const float maxError = .00001f) const {
        auto m1 = _domain->clone(), m2 = _domain->clone();
        auto d1 = _range->clone(), d2 = _range->clone();
        m1->random();
        d1->random();
        forward(false, m1, d2);
        adjoint(false, m2, d1);
        const double a1 = gpuDot(d1, d2), b1 = gpuDot(m1, m2);
        const double eNoAdd = std::fabs((a1 - b1) / b1);
        forward(true, m1, d2);
        adjoint(true, m2, d1);
        const double a2 = gpuDot(d1, d2), b2 = gpuDot(m1, m2);
        const double eAdd = std::fabs((a2 - b2) / b2);
        if (verbose) {
            std::cout << std::setprecision(16) << "WITHOUT ADD: <F m, d> = " << a1 << ", <m, F* d> = " << b1
                      << ", relative error = " << eNoAdd << std::endl;
            std::cout << "WITH ADD: <F m, d> = " << a2 << ", <m, F* d> = " << b2 << ", relative error = " << eAdd
                      << std::endl;
        }
        return eNoAdd <= maxError && eAdd <= maxError;
    }

    // GPU of the dot-product test's reductions (the shot operators: their first GPU), or -1 for
    // host reductions (host operators such as deviceGpu)
    virtual int dotTestDevice() const { return -1; }

    void setDomainRange(const std::shared_ptr<V1> dom, const std::shared_ptr<V2> rng) {
        _domain = dom->cloneSpace();
        _range = rng->cloneSpace();
    }
    std::shared_ptr<V1> getDomain() { return _domain; }
    std::shared_ptr<V2> getRange() { return _range; }

  protected:
    Operator() = default;

    template <class V>
    double gpuDot(const std::shared_ptr<V>& a, const std::shared_ptr<V>& b) const {
        if (dotTestDevice() < 0) return a->dot(b);
        double r = 0.0;
        const long long n = a->getHyper()->getN123();
        if (n != b->getHyper()->getN123()) throw std::runtime_error("dotTest: vectors of different sizes");
        if (aio_dot_f64(dotTestDevice(), AIO_MEM_HOST, n, a->getVals(), b->getVals(), &r) != AIO_OK)
            throw std::runtime_error("dotTest: FP64 reduction on the GPU failed");
        return r;
    }

  private:
    std::shared_ptr<V1> _domain;
    std::shared_ptr<V2> _range;
};
