// Linear operator interface of the reference (F/include/operator.h:7-100):
// forward(add, model, data) / adjoint(add, model, data), where add = false
// overwrites the output and add = true accumulates into it; a domain / range
// pair set by setDomainRange; and the dot-product test.
#pragma once
#include <cmath>
#include <iomanip>
#include <iostream>
#include <memory>

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
    // error of each pair must not exceed maxError. Dot products accumulate in FP64.
    bool dotTest(const bool verbose = false, const float maxError = .00001f) const {
        auto m1 = _domain->clone(), m2 = _domain->clone();
        auto d1 = _range->clone(), d2 = _range->clone();
        m1->random();
        d1->random();
        forward(false, m1, d2);
        adjoint(false, m2, d1);
        const double a1 = d1->dot(d2), b1 = m1->dot(m2);
        const double eNoAdd = std::fabs((a1 - b1) / b1);
        forward(true, m1, d2);
        adjoint(true, m2, d1);
        const double a2 = d1->dot(d2), b2 = m1->dot(m2);
        const double eAdd = std::fabs((a2 - b2) / b2);
        if (verbose) {
            std::cout << std::setprecision(16) << "WITHOUT ADD: <F m, d> = " << a1 << ", <m, F* d> = " << b1
                      << ", relative error = " << eNoAdd << std::endl;
            std::cout << "WITH ADD: <F m, d> = " << a2 << ", <m, F* d> = " << b2 << ", relative error = " << eAdd
                      << std::endl;
        }
        return eNoAdd <= maxError && eAdd <= maxError;
    }

    void setDomainRange(const std::shared_ptr<V1> dom, const std::shared_ptr<V2> rng) {
        _domain = dom->cloneSpace();
        _range = rng->cloneSpace();
    }
    std::shared_ptr<V1> getDomain() { return _domain; }
    std::shared_ptr<V2> getRange() { return _range; }

  protected:
    Operator() = default;

  private:
    std::shared_ptr<V1> _domain;
    std::shared_ptr<V2> _range;
};
