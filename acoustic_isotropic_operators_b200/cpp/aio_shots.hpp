// Reference-facing C++ operator classes over the B200 C ABI (include/aio_b200.h).
//
// Same public constructors and methods as the reference's host classes
// (F/include/deviceGpu.h, fdParam.h, nonlinearPropShotsGpu.h, BornShotsGpu.h,
// BornExtShotsGpu.h, tomoExtShotsGpu.h, wemvaExtShotsGpu.h), same parameter keys,
// same host-side numerics (device spread / gather, d2/dt2, dtw^2 v^2 scaling,
// linear time interpolation), same error type (std::runtime_error). What differs
// is the schedule: the reference runs one shot per GPU at a time through an
// OpenMP loop; here every shot assigned to a GPU goes to that GPU's engine
// context in ONE batched call (the engine runs them together), one host thread
// per GPU of the list, and per-GPU images are summed on the host.
//
// Header-only; link with libaio_b200.so.
#pragma once
#include <algorithm>
#include <cmath>
#include <iostream>
#include <numeric>
#include <thread>
#include <unordered_map>

#include "aio_b200.h"
#include "aio_operator.hpp"
#include "aio_sep.hpp"

namespace aio_ops {

inline void ck(int rc) {
    if (rc != AIO_OK) throw std::runtime_error(std::string("acoustic_isotropic_operators_b200: ") + aio_last_error());
}
inline void fail(const std::string& m) {
    std::cout << "**** ERROR: " << m << " ****" << std::endl;
    throw std::runtime_error(m);
}

}  // namespace aio_ops

// --------------------------------------------------------------------------- deviceGpu
// Sources / receivers: each (irregular) device spreads onto the 4 grid corners
// around it (8 with a dipole), weights bilinear (constructor 1) or a single
// unit weight (constructors 2, 3: devices on grid points). Traces on the grid
// ("regular") are indexed by the unique excited grid points in order of first
// appearance (F/src/deviceGpu.cpp:8-261).
class deviceGpu : public Operator<SEP::float2DReg, SEP::float2DReg> {
  public:
    // #1: physical coordinates (same units as the velocity axes)
    deviceGpu(const std::shared_ptr<SEP::float1DReg> zCoord, const std::shared_ptr<SEP::float1DReg> xCoord,
              const std::shared_ptr<SEP::float2DReg> vel, int& nt, int dipole, float zDipoleShift,
              float xDipoleShift)
        : _nt(nt), _nbCorner(dipole == 1 ? 8 : 4) {
        const SEP::axis az = vel->getHyper()->getAxis(1), ax = vel->getHyper()->getAxis(2);
        _nz = az.n;
        _nDeviceIrreg = zCoord->getHyper()->getAxis(1).n;
        const float zMax = az.o + (az.n - 1) * az.d, xMax = ax.o + (ax.n - 1) * ax.d;
        for (int i = 0; i < _nDeviceIrreg; i++)
            if ((*zCoord->_mat)[i] >= zMax || (*xCoord->_mat)[i] >= xMax) aio_ops::fail("One of the device is out of bounds");
        _idx.resize((size_t)_nbCorner * _nDeviceIrreg);
        _w.resize(_idx.size());
        for (int i = 0; i < _nDeviceIrreg; i++) {
            bilinear(i * _nbCorner, (*zCoord->_mat)[i], (*xCoord->_mat)[i], az, ax, 1.0);
            if (_nbCorner == 8)
                bilinear(i * _nbCorner + 4, (*zCoord->_mat)[i] + zDipoleShift, (*xCoord->_mat)[i] + xDipoleShift, az,
                         ax, -1.0);
        }
        unique();
    }
    // #2: grid indices per device
    deviceGpu(const std::vector<int>& zGridVector, const std::vector<int>& xGridVector,
              const std::shared_ptr<SEP::float2DReg> vel, int& nt, int dipole, int zDipoleShift, int xDipoleShift)
        : _nt(nt), _nbCorner(dipole == 1 ? 8 : 4) {
        _nz = vel->getHyper()->getAxis(1).n;
        _nDeviceIrreg = (int)zGridVector.size();
        if (zGridVector.size() != xGridVector.size()) aio_ops::fail("z and x device lists differ in length");
        const int zMax = *std::max_element(zGridVector.begin(), zGridVector.end());
        const int xMax = *std::max_element(xGridVector.begin(), xGridVector.end());
        if (zMax >= _nz || xMax >= vel->getHyper()->getAxis(2).n) aio_ops::fail("One of the device is out of bounds");
        _idx.resize((size_t)_nbCorner * _nDeviceIrreg);
        _w.resize(_idx.size());
        for (int i = 0; i < _nDeviceIrreg; i++) {
            onGrid(i * _nbCorner, xGridVector[i] * _nz + zGridVector[i], 1.f);
            if (_nbCorner == 8)
                onGrid(i * _nbCorner + 4, (xGridVector[i] + xDipoleShift) * _nz + zGridVector[i] + zDipoleShift, -1.f);
        }
        unique();
    }
    // #3: a regular z-x array of devices on the grid
    deviceGpu(const int& nzDevice, const int& ozDevice, const int& dzDevice, const int& nxDevice, const int& oxDevice,
              const int& dxDevice, const std::shared_ptr<SEP::float2DReg> vel, int& nt, int dipole, int zDipoleShift,
              int xDipoleShift)
        : _nt(nt), _nbCorner(dipole == 1 ? 8 : 4) {
        _nz = vel->getHyper()->getAxis(1).n;
        _nDeviceIrreg = nzDevice * nxDevice;
        if (ozDevice + (nzDevice - 1) * dzDevice >= _nz || oxDevice + (nxDevice - 1) * dxDevice >= vel->getHyper()->getAxis(2).n)
            aio_ops::fail("One of the device is out of bounds");
        _idx.resize((size_t)_nbCorner * _nDeviceIrreg);
        _w.resize(_idx.size());
        int d = 0;
        for (int ix = 0; ix < nxDevice; ix++)
            for (int iz = 0; iz < nzDevice; iz++, d++) {
                const int gx = oxDevice + ix * dxDevice, gz = ozDevice + iz * dzDevice;
                onGrid(d * _nbCorner, gx * _nz + gz, 1.f);
                if (_nbCorner == 8) onGrid(d * _nbCorner + 4, (gx + xDipoleShift) * _nz + gz + zDipoleShift, -1.f);
            }
        unique();
    }

    // Windowed-sinc devices (Hicks 2002, "Arbitrary source and receiver positioning in
    // finite-difference schemes using Kaiser windowed sinc functions", Geophysics 67(1)):
    // each device at physical coordinates spreads onto the (2r)^2 grid points around it
    // with weights wz(iz) * wx(ix), w(i) = sinc(i - p) * K(i - p), p the coordinate in grid
    // units, K(x) = I0(beta * sqrt(1 - (x/r)^2)) / I0(beta) the Kaiser window of half-width
    // r = halfWidth. On a grid node the weights reduce to the node (sinc vanishes at the
    // other integers). With a dipole the shifted point carries the negated weights. Not in
    // the reference (its devices are bilinear); every stencil point must lie on the grid.
    static std::shared_ptr<deviceGpu> windowedSinc(const std::shared_ptr<SEP::float1DReg> zCoord,
                                                   const std::shared_ptr<SEP::float1DReg> xCoord,
                                                   const std::shared_ptr<SEP::float2DReg> vel, int nt, int halfWidth = 4,
                                                   float beta = 4.14f, int dipole = 0, float zDipoleShift = 0.f,
                                                   float xDipoleShift = 0.f) {
        if (halfWidth < 1 || halfWidth > 10) aio_ops::fail("windowed sinc: half-width must be 1 to 10");
        const int w1 = 2 * halfWidth, nPt = w1 * w1;
        std::shared_ptr<deviceGpu> d(new deviceGpu(nt, (dipole == 1 ? 2 : 1) * nPt));
        const SEP::axis az = vel->getHyper()->getAxis(1), ax = vel->getHyper()->getAxis(2);
        d->_nz = az.n;
        d->_nDeviceIrreg = zCoord->getHyper()->getAxis(1).n;
        d->_idx.resize((size_t)d->_nbCorner * d->_nDeviceIrreg);
        d->_w.resize(d->_idx.size());
        auto weights1d = [&](double p, int n, int& first, double* w) {
            const int f = (int)std::floor(p);
            first = f - halfWidth + 1;
            if (first < 0 || first + w1 > n) aio_ops::fail("One of the device is out of bounds (windowed-sinc stencil)");
            const double pi = 3.14159265358979323846, i0b = besselI0(beta);
            for (int k = 0; k < w1; k++) {
                const double x = first + k - p;
                const double sinc = std::fabs(x) < 1e-12 ? 1.0 : std::sin(pi * x) / (pi * x);
                const double u = x / halfWidth;
                w[k] = std::fabs(u) <= 1.0 ? sinc * besselI0(beta * std::sqrt(1.0 - u * u)) / i0b : 0.0;
            }
        };
        auto point = [&](int i1, float zc, float xc, double sign) {
            double wz[20], wx[20];
            int z0, x0;
            weights1d(((double)zc - az.o) / az.d, az.n, z0, wz);
            weights1d(((double)xc - ax.o) / ax.d, ax.n, x0, wx);
            for (int jx = 0; jx < w1; jx++)
                for (int jz = 0; jz < w1; jz++) {
                    d->_idx[i1 + jx * w1 + jz] = (x0 + jx) * d->_nz + z0 + jz;
                    d->_w[i1 + jx * w1 + jz] = (float)(sign * wz[jz] * wx[jx]);
                }
        };
        for (int i = 0; i < d->_nDeviceIrreg; i++) {
            const float zc = (*zCoord->_mat)[i], xc = (*xCoord->_mat)[i];
            point(i * d->_nbCorner, zc, xc, 1.0);
            if (dipole == 1) point(i * d->_nbCorner + nPt, zc + zDipoleShift, xc + xDipoleShift, -1.0);
        }
        d->unique();
        return d;
    }
    // modified Bessel function of the first kind, order 0 (power series)
    static double besselI0(double x) {
        double sum = 1.0, term = 1.0;
        for (int k = 1; k < 60; k++) {
            term *= (x / (2.0 * k)) * (x / (2.0 * k));
            sum += term;
            if (term < 1e-17 * sum) break;
        }
        return sum;
    }

    // regular [nDeviceReg][nt] -> irregular [nDeviceIrreg][nt]
    void forward(const bool add, const std::shared_ptr<SEP::float2DReg> signalReg,
                 std::shared_ptr<SEP::float2DReg> signalIrreg) const override {
        aio_ops::ck(aio_device_gather(add ? 1 : 0, _nDeviceIrreg, _nbCorner, _trace.data(), _w.data(), _nDeviceReg,
                                      signalReg->getHyper()->getAxis(1).n, signalReg->getVals(), signalIrreg->getVals()));
    }
    // irregular -> regular
    void adjoint(const bool add, std::shared_ptr<SEP::float2DReg> signalReg,
                 const std::shared_ptr<SEP::float2DReg> signalIrreg) const override {
        aio_ops::ck(aio_device_spread(add ? 1 : 0, _nDeviceIrreg, _nbCorner, _trace.data(), _w.data(), _nDeviceReg,
                                      signalIrreg->getHyper()->getAxis(1).n, signalIrreg->getVals(), signalReg->getVals()));
    }

    int* getRegPosUnique() { return _unique.data(); }
    int* getRegPos() { return _idx.data(); }
    int getNt() { return _nt; }
    int getNDeviceReg() { return _nDeviceReg; }
    int getNDeviceIrreg() { return _nDeviceIrreg; }
    float* getWeights() { return _w.data(); }
    int getSizePosUnique() { return (int)_unique.size(); }
    // corner -> regular trace index (input of the C ABI spread / gather helpers)
    const int* cornerTraces() const { return _trace.data(); }
    int nCorner() const { return _nbCorner; }

  private:
    deviceGpu(int nt, int nCorner) : _nt(nt), _nbCorner(nCorner) {}
    // Same float / double expression sequence as the reference's constructor #1.
    void bilinear(int i1, float zc, float xc, const SEP::axis& az, const SEP::axis& ax, double sign) {
        float wz = (zc - az.o) / az.d;
        float wx = (xc - ax.o) / ax.d;
        const int zReg = wz;
        wz = wz - zReg;
        wz = 1.0 - wz;
        const int xReg = wx;
        wx = wx - xReg;
        wx = 1.0 - wx;
        _idx[i1] = xReg * _nz + zReg;
        _idx[i1 + 1] = _idx[i1] + 1;
        _idx[i1 + 2] = _idx[i1] + _nz;
        _idx[i1 + 3] = _idx[i1] + _nz + 1;
        if (sign > 0) {
            _w[i1] = wz * wx;
            _w[i1 + 1] = (1.0 - wz) * wx;
            _w[i1 + 2] = wz * (1.0 - wx);
            _w[i1 + 3] = (1.0 - wz) * (1.0 - wx);
        } else {
            _w[i1] = (-1.0) * wz * wx;
            _w[i1 + 1] = (-1.0) * (1.0 - wz) * wx;
            _w[i1 + 2] = (-1.0) * wz * (1.0 - wx);
            _w[i1 + 3] = (-1.0) * (1.0 - wz) * (1.0 - wx);
        }
    }
    void onGrid(int i1, int idx, float w0) {
        _idx[i1] = idx;
        _idx[i1 + 1] = idx + 1;
        _idx[i1 + 2] = idx + _nz;
        _idx[i1 + 3] = idx + _nz + 1;
        _w[i1] = w0;
        _w[i1 + 1] = _w[i1 + 2] = _w[i1 + 3] = 0.f;
    }
    void unique() {
        std::unordered_map<int, int> seen;
        _trace.resize(_idx.size());
        for (size_t i = 0; i < _idx.size(); i++) {
            auto it = seen.find(_idx[i]);
            if (it == seen.end()) {
                it = seen.emplace(_idx[i], (int)_unique.size()).first;
                _unique.push_back(_idx[i]);
            }
            _trace[i] = it->second;
        }
        _nDeviceReg = (int)_unique.size();
    }

    int _nt, _nbCorner, _nz = 0, _nDeviceIrreg = 0, _nDeviceReg = 0;
    std::vector<int> _idx, _trace, _unique;
    std::vector<float> _w;
};

// --------------------------------------------------------------------------- fdParam
// Parameter-file reading and checks of the reference (F/src/fdParam.cpp:9-139,
// 228-300): coarse / fine time axes, padding, sponge width minPad, extension,
// stability (Courant <= 0.45) and dispersion (>= 3 points per minimum
// wavelength) checks on the interior velocity, interior extents multiples of
// blockSize, and the propagation fields v^2 dtw^2 and 2 / v^3.
class fdParam {
  public:
    fdParam(const std::shared_ptr<SEP::float2DReg> vel, const std::shared_ptr<paramObj> par) : _vel(vel), _par(par) {
        _nts = par->getInt("nts");
        _dts = par->getFloat("dts", 0.0f);
        _ots = par->getFloat("ots", 0.0f);
        _sub = par->getInt("sub");
        _ntw = (_nts - 1) * _sub + 1;
        _dtw = _dts / float(_sub);
        _nz = par->getInt("nz");
        _freeSurface = par->getInt("freeSurface", 0);
        _zPadPlus = par->getInt("zPadPlus");
        _zPadMinus = par->getInt("zPadMinus");
        _zPad = _freeSurface == 1 ? _zPadPlus : std::min(_zPadMinus, _zPadPlus);
        _dz = par->getFloat("dz", -1.0f);
        _oz = vel->getHyper()->getAxis(1).o;
        if ((_zPadMinus == 0 && _freeSurface != 1) || (_zPadMinus > 0 && _freeSurface == 1))
            aio_ops::fail("[fdParam]: zPadMinus and freeSurface flag are inconsistent");
        if (_nz != vel->getHyper()->getAxis(1).n) aio_ops::fail("[fdParam]: nz from vel tag not consistent with nz from parfile");
        _nx = par->getInt("nx");
        _xPadPlus = par->getInt("xPadPlus");
        _xPadMinus = par->getInt("xPadMinus");
        _xPad = std::min(_xPadMinus, _xPadPlus);
        _dx = par->getFloat("dx", -1.0f);
        _ox = vel->getHyper()->getAxis(2).o;
        if (_nx != vel->getHyper()->getAxis(2).n) aio_ops::fail("[fdParam]: nx from vel tag not consistent with nx from parfile");
        _nExt = par->getInt("nExt", 1);
        if (_nExt % 2 == 0) aio_ops::fail("Length of extended axis must be an uneven number");
        _hExt = (_nExt - 1) / 2;
        _extension = par->getString("extension", "none");
        _fMax = par->getFloat("fMax", 1000.0f);
        _blockSize = par->getInt("blockSize");
        _fat = par->getInt("fat");
        if (_fat != 5) aio_ops::fail("fat must be 5 (10th-order stencil)");
        _minPad = std::min(_zPad, _xPad);
        _saveWavefield = par->getInt("saveWavefield", 0);
        _alphaCos = par->getFloat("alphaCos", 0.99f);
        _errorTolerance = par->getFloat("errorTolerance", 0.000001f);
        if (std::abs(_dz - vel->getHyper()->getAxis(1).d) > _errorTolerance ||
            std::abs(_dx - vel->getHyper()->getAxis(2).d) > _errorTolerance)
            aio_ops::fail("[Velocity file] dz / dx not consistent with parfile");
        // interior velocity extrema (the FAT ring excluded)
        float vmin = INFINITY, vmax = -INFINITY;
        for (int ix = _fat; ix < _nx - _fat; ix++)
            for (int iz = _fat; iz < _nz - _fat; iz++) {
                const float v = (*vel->_mat)[ix][iz];
                vmin = std::min(vmin, v);
                vmax = std::max(vmax, v);
            }
        _maxVel = vmax;
        _minVel = vmin;
        _Courant = _maxVel * _dtw / std::min(_dz, _dx);
        if (_Courant > 0.45f) aio_ops::fail("Courant is too big: " + std::to_string(_Courant));
        _dispersionRatio = _minVel / (_fMax * std::max(_dz, _dx));
        if (_dispersionRatio < 3.0f) aio_ops::fail("Dispersion is too small: " + std::to_string(_dispersionRatio));
        if ((_nz - 2 * _fat) % _blockSize != 0) aio_ops::fail("nz not a multiple of block size");
        if ((_nx - 2 * _fat) % _blockSize != 0) aio_ops::fail("nx not a multiple of block size");
        _vel2Dtw2.resize((size_t)_nz * _nx);
        _reflectivityScale.resize(_vel2Dtw2.size());
        aio_ops::ck(aio_fd_precompute(_nz, _nx, _dts, _sub, vel->getVals(), _vel2Dtw2.data(), _reflectivityScale.data()));
    }

    bool checkParfileConsistencyTime(const std::shared_ptr<SEP::float2DReg> traces, int timeAxisIndex,
                                     const std::string& what) const {
        const SEP::axis a = traces->getHyper()->getAxis(timeAxisIndex);
        if (_nts != a.n || std::abs(_dts - a.d) > _errorTolerance || std::abs(_ots - a.o) > _errorTolerance) {
            std::cout << "**** [" << what << "] ERROR: time axis not consistent with parfile ****" << std::endl;
            return false;
        }
        return true;
    }
    template <class V>
    bool checkParfileConsistencySpace(const std::shared_ptr<V> m, const std::string& what) const {
        const SEP::axis az = m->getHyper()->getAxis(1), ax = m->getHyper()->getAxis(2);
        if (_nz != az.n || _nx != ax.n || std::abs(_dz - az.d) > _errorTolerance || std::abs(_dx - ax.d) > _errorTolerance ||
            std::abs(_oz - az.o) > _errorTolerance || std::abs(_ox - ax.o) > _errorTolerance) {
            std::cout << "**** [" << what << "] ERROR: space axes not consistent with parfile ****" << std::endl;
            return false;
        }
        return true;
    }

    aio_params engineParams(int device, int leg1 = 1, int leg2 = 1) const {
        aio_params p{};
        p.nz = _nz;
        p.nx = _nx;
        p.nts = _nts;
        p.sub = _sub;
        p.minPad = _minPad;
        p.nExt = _nExt;
        p.dz = _dz;
        p.dx = _dx;
        p.dts = _dts;
        p.alphaCos = _alphaCos;
        p.leg1 = leg1;
        p.leg2 = leg2;
        p.sloth = 0;
        p.wavefieldPrecision = AIO_WFLD_FP32;
        p.imageFp64 = 1;
        p.device = device;
        p.memBudgetBytes = 0;
        p.stepper = AIO_STEPPER_AUTO;
        p.chunkColumns = 0;
        p.freeSurface = _freeSurface;
        // time-lag or subsurface-offset drivers of the extended classes (F/src/BornExtGpu.cpp:41-59)
        p.extension = _extension == "offset" ? AIO_EXT_OFFSET : AIO_EXT_TIME;
        return p;
    }

    std::shared_ptr<SEP::float2DReg> _vel;
    std::shared_ptr<paramObj> _par;
    int _nts, _sub, _ntw, _nz, _nx, _freeSurface, _zPadPlus, _zPadMinus, _zPad, _xPadPlus, _xPadMinus, _xPad;
    int _nExt, _hExt, _blockSize, _fat, _minPad, _saveWavefield;
    float _dts, _ots, _dtw, _dz, _dx, _oz, _ox, _fMax, _alphaCos, _errorTolerance;
    float _maxVel, _minVel, _Courant, _dispersionRatio;
    std::string _extension;
    std::vector<float> _vel2Dtw2, _reflectivityScale;
};

// --------------------------------------------------------------------------- shot loop
namespace aio_ops {

// Prepared per-shot geometry and signals on the unique grid points.
struct PreparedShot {
    std::vector<int> srcPos, recPos;
    std::vector<float> srcFine;   // [nSrcReg][ntw]
    std::vector<float> dataReg;   // [nRecReg][nts]
    std::vector<float> wemvaReg;  // [nRecReg][nts]
    std::vector<float> srcOut;    // nonlinear adjoint: [nSrcReg][ntw]
};

// Shared machinery of the five shot-loop classes: parameter keys nShot, nGpu,
// iGpu, info, deviceNumberInfo, saveWavefield, wavefieldShotNumber; GPU list
// rules of the reference (F/src/BornShotsGpu.cpp:26-57); one engine context per
// GPU of the list, created on first use and refreshed by setVel.
class ShotLoop {
  public:
    ShotLoop(std::shared_ptr<SEP::float2DReg> vel, std::shared_ptr<paramObj> par, int family)
        : _vel(vel), _par(par), _family(family) {
        _nShot = par->getInt("nShot");
        createGpuIdList();
        _info = par->getInt("info", 0);
        _deviceNumberInfo = par->getInt("deviceNumberInfo", _gpuList[0]);
        ck(aio_getGpuInfo(_gpuList.data(), (int)_gpuList.size(), _info, _deviceNumberInfo));
        _saveWavefield = par->getInt("saveWavefield", 0);
        _wavefieldShotNumber = par->getInt("wavefieldShotNumber", 0);
        _leg1 = par->getInt("leg1", 1);
        _sloth = par->getInt("sloth", 0);  // F/src/BornExtGpu.cpp:14, F/src/tomoExtGpu.cpp:15
        _leg2 = par->getInt("leg2", 1);
    }
    virtual ~ShotLoop() { release(); }

    void createGpuIdList() {
        _nGpu = _par->getInt("nGpu", -1);
        _gpuList = _par->getInts("iGpu", std::vector<int>{-1});
        if (_nGpu <= 0 && _gpuList[0] < 0) fail("Please provide a list of GPUs to be used");
        if (_nGpu > 0 && _gpuList[0] < 0) {
            _gpuList.clear();
            for (int i = 0; i < _nGpu; i++) _gpuList.push_back(i);
        }
        if (_gpuList[0] >= 0) {
            _nGpu = (int)_gpuList.size();
            std::sort(_gpuList.begin(), _gpuList.end());
            if (std::adjacent_find(_gpuList.begin(), _gpuList.end()) != _gpuList.end())
                fail("Please make sure there are no duplicates in the list");
        }
    }
    void setVelocity(std::shared_ptr<SEP::float2DReg> vel) {
        _vel = vel;
        release();
    }

  protected:
    const fdParam& fd() const {
        if (!_fd) _fd = std::make_shared<fdParam>(_vel, _par);
        return *_fd;
    }
    aio_context* context(int iGpu) const {
        if (_ctx.empty()) _ctx.assign(_gpuList.size(), nullptr);
        if (!_ctx[iGpu]) {
            const fdParam& f = fd();
            aio_params p = f.engineParams(_gpuList[iGpu], _leg1, _leg2);
            if (!_freeSurfaceDrivers) p.freeSurface = 0;
            // the free-surface drivers take no sloth flag (e.g. F/include/BornExtShotsGpuFunctions.h:27)
            p.sloth = p.freeSurface ? 0 : _sloth;
            ck(aio_context_create(&p, f._vel2Dtw2.data(), f._reflectivityScale.data(), &_ctx[iGpu]));
        }
        return _ctx[iGpu];
    }
    void release() {
        for (auto* c : _ctx)
            if (c) aio_context_destroy(c);
        _ctx.clear();
        _fd.reset();
    }
    // Shots of GPU i: a contiguous range (the engine batches them in one call).
    std::pair<int, int> range(int iGpu) const {
        const int per = (_nShot + _nGpu - 1) / _nGpu;
        return {std::min(_nShot, iGpu * per), std::min(_nShot, (iGpu + 1) * per)};
    }
    // Run fn(iGpu, first shot, end shot) on one host thread per GPU; rethrow the first error.
    template <class F>
    void perGpu(F fn) const {
        std::vector<std::string> errs(_nGpu);
        std::vector<std::thread> th;
        for (int g = 0; g < _nGpu; g++)
            th.emplace_back([&, g] {
                try {
                    auto r = range(g);
                    if (r.first < r.second) fn(g, r.first, r.second);
                } catch (const std::exception& e) {
                    errs[g] = e.what();
                }
            });
        for (auto& t : th) t.join();
        for (auto& e : errs)
            if (!e.empty()) throw std::runtime_error(e);
    }

    // Source chain of seismicOperator2D::setSources (F/include/seismicOperator2D.cpp:10-39):
    // spread to the grid, [d2/dt2], dtw^2 v^2 at the grid point, linear interpolation to fine time.
    void prepareSource(deviceGpu& src, const float* traces, bool secondDerivative, PreparedShot& s) const {
        const fdParam& f = fd();
        const int nReg = src.getNDeviceReg();
        s.srcPos.assign(src.getRegPosUnique(), src.getRegPosUnique() + nReg);
        std::vector<float> reg((size_t)nReg * f._nts), d2;
        ck(aio_device_spread(0, src.getNDeviceIrreg(), src.nCorner(), src.cornerTraces(), src.getWeights(), nReg, f._nts,
                             traces, reg.data()));
        float* cur = reg.data();
        if (secondDerivative) {
            d2.resize(reg.size());
            ck(aio_second_time_derivative(0, f._nts, f._dts, nReg, reg.data(), d2.data()));
            cur = d2.data();
        }
        ck(aio_scale_seismic_source(nReg, s.srcPos.data(), f._nts, f._dts, f._sub, _vel->getVals(), cur));
        s.srcFine.assign((size_t)nReg * f._ntw, 0.f);
        ck(aio_time_interp_forward(0, f._nts, f._dts, f._ots, f._sub, nReg, cur, s.srcFine.data()));
    }
    void prepareReceivers(deviceGpu& rec, PreparedShot& s) const {
        s.recPos.assign(rec.getRegPosUnique(), rec.getRegPosUnique() + rec.getNDeviceReg());
        s.dataReg.assign((size_t)rec.getNDeviceReg() * fd()._nts, 0.f);
    }
    static aio_shot toShot(PreparedShot& s) {
        aio_shot a{};
        a.sourcesPositionReg = s.srcPos.data();
        a.nSourcesReg = (int)s.srcPos.size();
        a.receiversPositionReg = s.recPos.data();
        a.nReceiversReg = (int)s.recPos.size();
        a.sourcesSignals = s.srcFine.empty() ? nullptr : s.srcFine.data();
        a.data = s.dataReg.data();
        a.wemvaData = s.wemvaReg.empty() ? nullptr : s.wemvaReg.data();
        a.sourcesOut = s.srcOut.empty() ? nullptr : s.srcOut.data();
        return a;
    }
    // data[iShot] (+)= gather(regular data) for shots [s0, s1)
    void gatherData(std::vector<std::shared_ptr<deviceGpu>>& recV, int s0, int s1, std::vector<PreparedShot>& ps,
                    const std::shared_ptr<SEP::float3DReg>& data) const {
        const int nts = fd()._nts, nRecIrreg = data->getHyper()->getAxis(2).n;
        for (int i = s0; i < s1; i++) {
            deviceGpu& rec = *recV[recIndex(recV, i)];
            ck(aio_device_gather(1, rec.getNDeviceIrreg(), rec.nCorner(), rec.cornerTraces(), rec.getWeights(),
                                 rec.getNDeviceReg(), nts, ps[i - s0].dataReg.data(),
                                 data->getVals() + (size_t)i * nRecIrreg * nts));
        }
    }
    void spreadData(std::vector<std::shared_ptr<deviceGpu>>& recV, int i, const float* irreg, std::vector<float>& reg) const {
        deviceGpu& rec = *recV[recIndex(recV, i)];
        reg.assign((size_t)rec.getNDeviceReg() * fd()._nts, 0.f);
        ck(aio_device_spread(0, rec.getNDeviceIrreg(), rec.nCorner(), rec.cornerTraces(), rec.getWeights(),
                             rec.getNDeviceReg(), fd()._nts, irreg, reg.data()));
    }
    // Receiver geometry of shot iShot. The reference's Born-family shot loops use the first
    // receiver geometry whenever the source signals are per shot, even with per-shot
    // receivers (F/src/BornShotsGpu.cpp:119-121 and the same branch in the extended, tomo
    // and WEMVA loops); _recFirst reproduces that selection.
    int recIndex(const std::vector<std::shared_ptr<deviceGpu>>& v, int iShot) const {
        return (v.size() == 1 || _recFirst) ? 0 : iShot;
    }
    static int sigIndex(size_t nSig, int iShot) { return nSig == 1 ? 0 : iShot; }

    std::shared_ptr<SEP::float2DReg> _vel;
    std::shared_ptr<paramObj> _par;
    int _family, _nShot = 0, _nGpu = 0, _info = 0, _deviceNumberInfo = 0, _saveWavefield = 0, _wavefieldShotNumber = 0;
    int _leg1 = 1, _leg2 = 1, _sloth = 0;
    // the family has free-surface drivers (the reference's WEMVA runs its plain drivers whatever
    // freeSurface says: F/src/wemvaExtGpu.cpp has no free-surface branch)
    bool _freeSurfaceDrivers = true;
    bool _recFirst = false;
    std::vector<int> _gpuList;
    mutable std::shared_ptr<fdParam> _fd;
    mutable std::vector<aio_context*> _ctx;
};

}  // namespace aio_ops

// Nonlinear propagation: model [nShot|1][nSrcIrreg][nts] -> data [nShot][nRecIrreg][nts]
// (F/src/nonlinearPropShotsGpu.cpp, F/src/nonlinearPropGpu.cpp).
class nonlinearPropShotsGpu : public Operator<SEP::float3DReg, SEP::float3DReg>, public aio_ops::ShotLoop {
  public:
    // the dot-product test reduces on the first GPU of the operator's list
    int dotTestDevice() const override { return _gpuList.empty() || _gpuList[0] < 0 ? 0 : _gpuList[0]; }
    nonlinearPropShotsGpu(std::shared_ptr<SEP::float2DReg> vel, std::shared_ptr<paramObj> par,
                          std::vector<std::shared_ptr<deviceGpu>> sourcesVector,
                          std::vector<std::shared_ptr<deviceGpu>> receiversVector)
        : ShotLoop(vel, par, AIO_NONLINEAR), _sourcesVector(sourcesVector), _receiversVector(receiversVector) {}

    void forward(const bool add, const std::shared_ptr<SEP::float3DReg> model,
                 std::shared_ptr<SEP::float3DReg> data) const override {
        run(add, model, data, nullptr);
    }
    void forwardWavefield(const bool add, const std::shared_ptr<SEP::float3DReg> model,
                          std::shared_ptr<SEP::float3DReg> data) {
        _wavefield = makeWavefield();
        run(add, model, data, _wavefield->getVals());
    }
    void adjoint(const bool add, std::shared_ptr<SEP::float3DReg> model,
                 const std::shared_ptr<SEP::float3DReg> data) const override {
        runAdj(add, model, data, nullptr);
    }
    void adjointWavefield(const bool add, std::shared_ptr<SEP::float3DReg> model,
                          const std::shared_ptr<SEP::float3DReg> data) {
        _wavefield = makeWavefield();
        runAdj(add, model, data, _wavefield->getVals());
    }
    std::shared_ptr<SEP::float3DReg> getWavefield() { return _wavefield; }
    void setVel(std::shared_ptr<SEP::float2DReg> vel) { setVelocity(vel); }

  private:
    std::shared_ptr<SEP::float3DReg> makeWavefield() const {
        const fdParam& f = fd();
        return std::make_shared<SEP::float3DReg>(SEP::axis(f._nz, f._oz, f._dz), SEP::axis(f._nx, f._ox, f._dx),
                                                 SEP::axis(f._nts, f._ots, f._dts));
    }
    void run(bool add, const std::shared_ptr<SEP::float3DReg>& model, const std::shared_ptr<SEP::float3DReg>& data,
             float* wavefield) const {
        if (!add) data->scale(0.0);
        const fdParam& f = fd();
        const int nSrcIrreg = model->getHyper()->getAxis(2).n;
        const bool constSrc = model->getHyper()->getAxis(3).n == 1;
        perGpu([&](int g, int s0, int s1) {
            std::vector<aio_ops::PreparedShot> ps(s1 - s0);
            std::vector<aio_shot> shots;
            for (int i = s0; i < s1; i++) {
                auto& s = ps[i - s0];
                const float* tr = model->getVals() + (size_t)(constSrc ? 0 : i) * nSrcIrreg * f._nts;
                prepareSource(*_sourcesVector[i], tr, false, s);
                prepareReceivers(*_receiversVector[recIndex(_receiversVector, i)], s);
                shots.push_back(toShot(s));
            }
            aio_context* c = context(g);
            for (int i = s0; i < s1; i++)
                if (wavefield && i == _wavefieldShotNumber) {
                    aio_ops::ck(aio_nonlinear_forward_wavefield(c, &shots[i - s0], AIO_MEM_HOST, wavefield));
                    shots[i - s0].nSourcesReg = -1;  // done
                }
            std::vector<aio_shot> rest;
            for (auto& a : shots)
                if (a.nSourcesReg >= 0) rest.push_back(a);
            if (!rest.empty()) aio_ops::ck(aio_nonlinear_forward(c, (int)rest.size(), rest.data(), AIO_MEM_HOST));
            gatherData(const_cast<std::vector<std::shared_ptr<deviceGpu>>&>(_receiversVector), s0, s1, ps, data);
        });
    }
    void runAdj(bool add, const std::shared_ptr<SEP::float3DReg>& model, const std::shared_ptr<SEP::float3DReg>& data,
                float* wavefield) const {
        if (!add) model->scale(0.0);
        const fdParam& f = fd();
        const int nSrcIrreg = model->getHyper()->getAxis(2).n;
        const bool constSrc = model->getHyper()->getAxis(3).n == 1;
        const int nRecIrreg = data->getHyper()->getAxis(2).n;
        std::vector<std::vector<float>> out(_nShot);
        perGpu([&](int g, int s0, int s1) {
            std::vector<aio_ops::PreparedShot> ps(s1 - s0);
            std::vector<aio_shot> shots;
            for (int i = s0; i < s1; i++) {
                auto& s = ps[i - s0];
                deviceGpu& src = *_sourcesVector[i];
                s.srcPos.assign(src.getRegPosUnique(), src.getRegPosUnique() + src.getNDeviceReg());
                s.recPos.assign(_receiversVector[recIndex(_receiversVector, i)]->getRegPosUnique(),
                                _receiversVector[recIndex(_receiversVector, i)]->getRegPosUnique() +
                                    _receiversVector[recIndex(_receiversVector, i)]->getNDeviceReg());
                spreadData(const_cast<std::vector<std::shared_ptr<deviceGpu>>&>(_receiversVector), i,
                           data->getVals() + (size_t)i * nRecIrreg * f._nts, s.dataReg);
                s.srcOut.assign((size_t)src.getNDeviceReg() * f._ntw, 0.f);
                shots.push_back(toShot(s));
            }
            aio_context* c = context(g);
            std::vector<aio_shot> rest;
            for (int i = s0; i < s1; i++) {
                if (wavefield && i == _wavefieldShotNumber)
                    aio_ops::ck(aio_nonlinear_adjoint_wavefield(c, &shots[i - s0], AIO_MEM_HOST, wavefield));
                else
                    rest.push_back(shots[i - s0]);
            }
            if (!rest.empty()) aio_ops::ck(aio_nonlinear_adjoint(c, (int)rest.size(), rest.data(), AIO_MEM_HOST));
            // fine -> coarse time, dtw^2 v^2, gather to the irregular sources (F/src/nonlinearPropGpu.cpp:82-111)
            for (int i = s0; i < s1; i++) {
                auto& s = ps[i - s0];
                deviceGpu& src = *_sourcesVector[i];
                const int nReg = src.getNDeviceReg();
                std::vector<float> coarse((size_t)nReg * f._nts);
                aio_ops::ck(aio_time_interp_adjoint(0, f._nts, f._dts, f._ots, f._sub, nReg, coarse.data(), s.srcOut.data()));
                aio_ops::ck(aio_scale_seismic_source(nReg, s.srcPos.data(), f._nts, f._dts, f._sub, _vel->getVals(), coarse.data()));
                out[i].assign((size_t)nSrcIrreg * f._nts, 0.f);
                aio_ops::ck(aio_device_gather(0, src.getNDeviceIrreg(), src.nCorner(), src.cornerTraces(), src.getWeights(), nReg,
                                              f._nts, coarse.data(), out[i].data()));
            }
        });
        for (int i = 0; i < _nShot; i++) {
            float* m = model->getVals() + (size_t)(constSrc ? 0 : i) * nSrcIrreg * f._nts;
            for (size_t k = 0; k < out[i].size(); k++) m[k] += out[i][k];
        }
        if (wavefield) {  // adjoint wavefield scaled by dtw^2 v^2 (F/src/nonlinearPropGpu.cpp:96-105)
            const float* v = _vel->getVals();
            const size_t n = (size_t)f._nz * f._nx;
            for (int t = 0; t < f._nts; t++)
                for (size_t k = 0; k < n; k++) wavefield[t * n + k] *= f._dtw * f._dtw * v[k] * v[k];
        }
    }

    std::vector<std::shared_ptr<deviceGpu>> _sourcesVector, _receiversVector;
    std::shared_ptr<SEP::float3DReg> _wavefield;
};

// Common body of the Born-family classes (model image shared by every shot).
namespace aio_ops {
template <class VM>
class BornFamily : public ShotLoop {
  public:
    BornFamily(std::shared_ptr<SEP::float2DReg> vel, std::shared_ptr<paramObj> par, int family,
               std::vector<std::shared_ptr<deviceGpu>> src, std::vector<std::shared_ptr<SEP::float2DReg>> sig,
               std::vector<std::shared_ptr<deviceGpu>> rec)
        : ShotLoop(vel, par, family), _sourcesVector(src), _sourcesSignalsVector(sig), _receiversVector(rec) {
        _recFirst = sig.size() != 1;
        // The reference's extended classes call their time-lag drivers for "time" and their
        // subsurface-offset ones for "offset"; any other value runs no driver in tomo, WEMVA and
        // the extended Born adjoint (F/src/tomoExtGpu.cpp:48-60, wemvaExtGpu.cpp:131-154,
        // BornExtGpu.cpp:95-124), so it is refused here.
        if (family == AIO_BORN_EXT || family == AIO_TOMO_EXT || family == AIO_WEMVA_EXT) {
            const std::string e = par->getString("extension", "none");
            if (e != "time" && e != "offset") fail("extension must be \"time\" or \"offset\" for the extended operators");
        }
    }

  protected:
    // Per GPU: prepare the shots [s0, s1) (sources, receivers, optional input data) and call body(ctx, shots).
    template <class Body>
    void forShots(const std::shared_ptr<SEP::float3DReg>* dataIn, bool wemvaData, Body body) const {
        const fdParam& f = fd();
        perGpu([&](int g, int s0, int s1) {
            std::vector<PreparedShot> ps(s1 - s0);
            std::vector<aio_shot> shots;
            for (int i = s0; i < s1; i++) {
                auto& s = ps[i - s0];
                prepareSource(*_sourcesVector[i], _sourcesSignalsVector[sigIndex(_sourcesSignalsVector.size(), i)]->getVals(),
                              true, s);
                prepareReceivers(*_receiversVector[recIndex(_receiversVector, i)], s);
                if (dataIn) {
                    const int nRecIrreg = (*dataIn)->getHyper()->getAxis(2).n;
                    spreadData(const_cast<std::vector<std::shared_ptr<deviceGpu>>&>(_receiversVector), i,
                               (*dataIn)->getVals() + (size_t)i * nRecIrreg * f._nts, s.dataReg);
                }
                if (wemvaData) {
                    auto& rs = *_receiversSignalsVector[sigIndex(_receiversSignalsVector.size(), i)];
                    spreadData(const_cast<std::vector<std::shared_ptr<deviceGpu>>&>(_receiversVector), i, rs.getVals(),
                               s.wemvaReg);
                }
                shots.push_back(toShot(s));
            }
            body(g, s0, s1, ps, shots);
        });
    }
    // Prepare shot i alone (sources, receivers, optional input data, optional WEMVA data) for a
    // one-shot call.
    aio_shot prepareOne(int i, const std::shared_ptr<SEP::float3DReg>* dataIn, PreparedShot& s,
                        bool wemvaData = false) const {
        const fdParam& f = fd();
        prepareSource(*_sourcesVector[i], _sourcesSignalsVector[sigIndex(_sourcesSignalsVector.size(), i)]->getVals(),
                      true, s);
        prepareReceivers(*_receiversVector[recIndex(_receiversVector, i)], s);
        if (dataIn) {
            const int nRecIrreg = (*dataIn)->getHyper()->getAxis(2).n;
            spreadData(const_cast<std::vector<std::shared_ptr<deviceGpu>>&>(_receiversVector), i,
                       (*dataIn)->getVals() + (size_t)i * nRecIrreg * f._nts, s.dataReg);
        }
        if (wemvaData) {
            auto& rs = *_receiversSignalsVector[sigIndex(_receiversSignalsVector.size(), i)];
            spreadData(const_cast<std::vector<std::shared_ptr<deviceGpu>>&>(_receiversVector), i, rs.getVals(),
                       s.wemvaReg);
        }
        if (s.dataReg.empty()) s.dataReg.assign((size_t)s.recPos.size() * f._nts, 0.f);
        return toShot(s);
    }
    // The three saved-wavefield containers of tomo and WEMVA, zero-filled (setAllWavefields(1)).
    void resetWavefields3() {
        _wSrc = coarseWavefield();
        _wSec1 = coarseWavefield();
        _wSec2 = coarseWavefield();
    }
    bool wavefieldShotValid() const {
        return _saveWavefield == 1 && _wavefieldShotNumber >= 0 && _wavefieldShotNumber < _nShot;
    }
    std::shared_ptr<SEP::float3DReg> _wSrc, _wSec1, _wSec2;
    // A coarse wavefield container [nts][nx][nz] (zeros), as the reference's setAllWavefields(1).
    std::shared_ptr<SEP::float3DReg> coarseWavefield() const {
        const fdParam& f = fd();
        return std::make_shared<SEP::float3DReg>(SEP::axis(f._nz, f._oz, f._dz), SEP::axis(f._nx, f._ox, f._dx),
                                                 SEP::axis(f._nts, f._ots, f._dts));
    }
    // out (+)= sum over GPUs of per-GPU partial images
    void sumImages(std::vector<std::vector<float>>& parts, float* out, size_t n, bool add) const {
        if (!add) std::fill(out, out + n, 0.f);
        for (auto& p : parts)
            if (!p.empty())
                for (size_t k = 0; k < n; k++) out[k] += p[k];
    }

    std::vector<std::shared_ptr<deviceGpu>> _sourcesVector;
    std::vector<std::shared_ptr<SEP::float2DReg>> _sourcesSignalsVector;
    std::vector<std::shared_ptr<deviceGpu>> _receiversVector;
    std::vector<std::shared_ptr<SEP::float2DReg>> _receiversSignalsVector;
};
}  // namespace aio_ops

// Born: model [nx][nz] -> data [nShot][nRecIrreg][nts] (F/src/BornShotsGpu.cpp, F/src/BornGpu.cpp).
class BornShotsGpu : public Operator<SEP::float2DReg, SEP::float3DReg>, public aio_ops::BornFamily<SEP::float2DReg> {
  public:
    // the dot-product test reduces on the first GPU of the operator's list
    int dotTestDevice() const override { return _gpuList.empty() || _gpuList[0] < 0 ? 0 : _gpuList[0]; }
    BornShotsGpu(std::shared_ptr<SEP::float2DReg> vel, std::shared_ptr<paramObj> par,
                 std::vector<std::shared_ptr<deviceGpu>> sourcesVector,
                 std::vector<std::shared_ptr<SEP::float2DReg>> sourcesSignalsVector,
                 std::vector<std::shared_ptr<deviceGpu>> receiversVector)
        : BornFamily(vel, par, AIO_BORN, sourcesVector, sourcesSignalsVector, receiversVector) {}

    void forward(const bool add, const std::shared_ptr<SEP::float2DReg> model,
                 std::shared_ptr<SEP::float3DReg> data) const override {
        if (!add) data->scale(0.0);
        forShots(nullptr, false, [&](int g, int s0, int s1, std::vector<aio_ops::PreparedShot>& ps, std::vector<aio_shot>& sh) {
            aio_ops::ck(aio_born_forward(context(g), model->getVals(), (int)sh.size(), sh.data(), AIO_MEM_HOST));
            gatherData(const_cast<std::vector<std::shared_ptr<deviceGpu>>&>(_receiversVector), s0, s1, ps, data);
        });
    }
    void adjoint(const bool add, std::shared_ptr<SEP::float2DReg> model,
                 const std::shared_ptr<SEP::float3DReg> data) const override {
        std::vector<std::vector<float>> parts(_nGpu);
        const size_t n = (size_t)model->size();
        forShots(&data, false, [&](int g, int, int, std::vector<aio_ops::PreparedShot>&, std::vector<aio_shot>& sh) {
            parts[g].assign(n, 0.f);
            aio_ops::ck(aio_born_adjoint(context(g), parts[g].data(), 0, (int)sh.size(), sh.data(), AIO_MEM_HOST));
        });
        sumImages(parts, model->getVals(), n, add);
    }
    // forward / adjoint of every shot, plus the coarse wavefields of shot wavefieldShotNumber when
    // saveWavefield = 1 (F/src/BornShotsGpu.cpp:145-340, F/src/BornGpu.cpp:37-50): source and
    // scattered wavefields (forward), the scaled receiver wavefield (adjoint); with
    // saveWavefield = 0 the reference returns zero-filled containers, and so does this class.
    void forwardWavefield(const bool add, const std::shared_ptr<SEP::float2DReg> model,
                          std::shared_ptr<SEP::float3DReg> data) {
        forward(add, model, data);
        _srcWavefield = coarseWavefield();
        _secWavefield = coarseWavefield();
        if (_saveWavefield != 1 || _wavefieldShotNumber < 0 || _wavefieldShotNumber >= _nShot) return;
        aio_ops::PreparedShot ps;
        aio_shot sh = prepareOne(_wavefieldShotNumber, nullptr, ps);
        std::vector<float> scratch((size_t)sh.nReceiversReg * fd()._nts);
        sh.data = scratch.data();
        aio_ops::ck(aio_born_forward_wavefield(context(0), model->getVals(), &sh, AIO_MEM_HOST,
                                               _srcWavefield->getVals(), _secWavefield->getVals()));
    }
    void adjointWavefield(const bool add, const std::shared_ptr<SEP::float2DReg> model,
                          std::shared_ptr<SEP::float3DReg> data) {
        adjoint(add, model, data);
        _srcWavefield = coarseWavefield();
        _secWavefield = coarseWavefield();
        if (_saveWavefield != 1 || _wavefieldShotNumber < 0 || _wavefieldShotNumber >= _nShot) return;
        aio_ops::PreparedShot ps;
        aio_shot sh = prepareOne(_wavefieldShotNumber, &data, ps);
        std::vector<float> image((size_t)model->size());
        // the reference's adjoint wavefield driver returns the receiver wavefield only: the source
        // wavefield container stays zero
        aio_ops::ck(aio_born_adjoint_wavefield(context(0), image.data(), 0, &sh, AIO_MEM_HOST, nullptr,
                                               _secWavefield->getVals()));
    }
    std::shared_ptr<SEP::float3DReg> getSrcWavefield() { return _srcWavefield; }
    std::shared_ptr<SEP::float3DReg> getSecWavefield() { return _secWavefield; }
    void setVel(std::shared_ptr<SEP::float2DReg> vel) { setVelocity(vel); }

  private:
    std::shared_ptr<SEP::float3DReg> _srcWavefield, _secWavefield;
};

// Extended (time-lag) Born: model [nExt][nx][nz] -> data (F/src/BornExtShotsGpu.cpp).
class BornExtShotsGpu : public Operator<SEP::float3DReg, SEP::float3DReg>, public aio_ops::BornFamily<SEP::float3DReg> {
  public:
    // the dot-product test reduces on the first GPU of the operator's list
    int dotTestDevice() const override { return _gpuList.empty() || _gpuList[0] < 0 ? 0 : _gpuList[0]; }
    BornExtShotsGpu(std::shared_ptr<SEP::float2DReg> vel, std::shared_ptr<paramObj> par,
                    std::vector<std::shared_ptr<deviceGpu>> sourcesVector,
                    std::vector<std::shared_ptr<SEP::float2DReg>> sourcesSignalsVector,
                    std::vector<std::shared_ptr<deviceGpu>> receiversVector)
        : BornFamily(vel, par, AIO_BORN_EXT, sourcesVector, sourcesSignalsVector, receiversVector) {}

    void forward(const bool add, const std::shared_ptr<SEP::float3DReg> model,
                 std::shared_ptr<SEP::float3DReg> data) const override {
        if (!add) data->scale(0.0);
        forShots(nullptr, false, [&](int g, int s0, int s1, std::vector<aio_ops::PreparedShot>& ps, std::vector<aio_shot>& sh) {
            aio_ops::ck(aio_born_ext_forward(context(g), model->getVals(), (int)sh.size(), sh.data(), AIO_MEM_HOST));
            gatherData(const_cast<std::vector<std::shared_ptr<deviceGpu>>&>(_receiversVector), s0, s1, ps, data);
        });
    }
    void adjoint(const bool add, std::shared_ptr<SEP::float3DReg> model,
                 const std::shared_ptr<SEP::float3DReg> data) const override {
        std::vector<std::vector<float>> parts(_nGpu);
        const size_t n = (size_t)model->size();
        forShots(&data, false, [&](int g, int, int, std::vector<aio_ops::PreparedShot>&, std::vector<aio_shot>& sh) {
            parts[g].assign(n, 0.f);
            aio_ops::ck(aio_born_ext_adjoint(context(g), parts[g].data(), 0, (int)sh.size(), sh.data(), AIO_MEM_HOST));
        });
        sumImages(parts, model->getVals(), n, add);
    }
    // forward / adjoint of every shot, plus the coarse wavefields of shot wavefieldShotNumber when
    // saveWavefield = 1 (F/src/BornExtShotsGpu.cpp:143-340, F/src/BornExtGpu.cpp:37-110): source and
    // scattered wavefields (forward), source and receiver wavefields (adjoint), computed like the
    // reference's *Wavefield drivers (non-sloth time-lag scaling); with saveWavefield = 0 the
    // containers stay zero-filled.
    void forwardWavefield(const bool add, const std::shared_ptr<SEP::float3DReg> model,
                          std::shared_ptr<SEP::float3DReg> data) {
        forward(add, model, data);
        _srcWavefield = coarseWavefield();
        _secWavefield = coarseWavefield();
        if (_saveWavefield != 1 || _wavefieldShotNumber < 0 || _wavefieldShotNumber >= _nShot) return;
        aio_ops::PreparedShot ps;
        aio_shot sh = prepareOne(_wavefieldShotNumber, nullptr, ps);
        std::vector<float> scratch((size_t)sh.nReceiversReg * fd()._nts);
        sh.data = scratch.data();
        aio_ops::ck(aio_born_ext_forward_wavefield(context(0), model->getVals(), &sh, AIO_MEM_HOST,
                                                   _srcWavefield->getVals(), _secWavefield->getVals()));
    }
    void adjointWavefield(const bool add, std::shared_ptr<SEP::float3DReg> model,
                          const std::shared_ptr<SEP::float3DReg> data) {
        adjoint(add, model, data);
        _srcWavefield = coarseWavefield();
        _secWavefield = coarseWavefield();
        if (_saveWavefield != 1 || _wavefieldShotNumber < 0 || _wavefieldShotNumber >= _nShot) return;
        aio_ops::PreparedShot ps;
        aio_shot sh = prepareOne(_wavefieldShotNumber, &data, ps);
        std::vector<float> image((size_t)model->size());
        aio_ops::ck(aio_born_ext_adjoint_wavefield(context(0), image.data(), 0, &sh, AIO_MEM_HOST,
                                                   _srcWavefield->getVals(), _secWavefield->getVals()));
    }
    std::shared_ptr<SEP::float3DReg> getSrcWavefield() { return _srcWavefield; }
    std::shared_ptr<SEP::float3DReg> getSecWavefield() { return _secWavefield; }
    std::shared_ptr<SEP::float2DReg> getVel() { return _vel; }
    void setVel(std::shared_ptr<SEP::float2DReg> vel) { setVelocity(vel); }

  private:
    std::shared_ptr<SEP::float3DReg> _srcWavefield, _secWavefield;
};

// Extended tomo: velocity perturbation [nx][nz] -> data, background extended reflectivity
// [nExt][nx][nz] (F/src/tomoExtShotsGpu.cpp).
class tomoExtShotsGpu : public Operator<SEP::float2DReg, SEP::float3DReg>, public aio_ops::BornFamily<SEP::float2DReg> {
  public:
    // the dot-product test reduces on the first GPU of the operator's list
    int dotTestDevice() const override { return _gpuList.empty() || _gpuList[0] < 0 ? 0 : _gpuList[0]; }
    tomoExtShotsGpu(std::shared_ptr<SEP::float2DReg> vel, std::shared_ptr<paramObj> par,
                    std::vector<std::shared_ptr<deviceGpu>> sourcesVector,
                    std::vector<std::shared_ptr<SEP::float2DReg>> sourcesSignalsVector,
                    std::vector<std::shared_ptr<deviceGpu>> receiversVector,
                    std::shared_ptr<SEP::float3DReg> reflectivityExt)
        : BornFamily(vel, par, AIO_TOMO_EXT, sourcesVector, sourcesSignalsVector, receiversVector),
          _reflectivityExt(reflectivityExt) {}

    void forward(const bool add, const std::shared_ptr<SEP::float2DReg> model,
                 std::shared_ptr<SEP::float3DReg> data) const override {
        if (!add) data->scale(0.0);
        forShots(nullptr, false, [&](int g, int s0, int s1, std::vector<aio_ops::PreparedShot>& ps, std::vector<aio_shot>& sh) {
            aio_ops::ck(aio_tomo_ext_forward(context(g), model->getVals(), _reflectivityExt->getVals(), (int)sh.size(),
                                             sh.data(), AIO_MEM_HOST));
            gatherData(const_cast<std::vector<std::shared_ptr<deviceGpu>>&>(_receiversVector), s0, s1, ps, data);
        });
    }
    void adjoint(const bool add, std::shared_ptr<SEP::float2DReg> model,
                 const std::shared_ptr<SEP::float3DReg> data) const override {
        std::vector<std::vector<float>> parts(_nGpu);
        const size_t n = (size_t)model->size();
        forShots(&data, false, [&](int g, int, int, std::vector<aio_ops::PreparedShot>&, std::vector<aio_shot>& sh) {
            parts[g].assign(n, 0.f);
            aio_ops::ck(aio_tomo_ext_adjoint(context(g), parts[g].data(), 0, _reflectivityExt->getVals(), (int)sh.size(),
                                             sh.data(), AIO_MEM_HOST));
        });
        sumImages(parts, model->getVals(), n, add);
    }
    // forward / adjoint of every shot, plus, with saveWavefield = 1, the saved wavefields of shot
    // wavefieldShotNumber (F/src/tomoExtShotsGpu.cpp:147-245, :343-440): d2/dt2 of the source
    // wavefield and the two secondary wavefields the drivers fill (forward: the last leg's first and
    // recorded scattered wavefields; adjoint: the receiver wavefield and the last leg's scattered
    // samples). With saveWavefield = 0 the containers stay zero-filled.
    void forwardWavefield(const bool add, const std::shared_ptr<SEP::float2DReg> model,
                          std::shared_ptr<SEP::float3DReg> data) {
        forward(add, model, data);
        resetWavefields3();
        if (!wavefieldShotValid()) return;
        aio_ops::PreparedShot ps;
        aio_shot sh = prepareOne(_wavefieldShotNumber, nullptr, ps);
        aio_ops::ck(aio_tomo_ext_forward_wavefield(context(0), model->getVals(), _reflectivityExt->getVals(), &sh,
                                                   AIO_MEM_HOST, _wSrc->getVals(), _wSec1->getVals(),
                                                   _wSec2->getVals()));
    }
    void adjointWavefield(const bool add, std::shared_ptr<SEP::float2DReg> model,
                          const std::shared_ptr<SEP::float3DReg> data) {
        adjoint(add, model, data);
        resetWavefields3();
        if (!wavefieldShotValid()) return;
        aio_ops::PreparedShot ps;
        aio_shot sh = prepareOne(_wavefieldShotNumber, &data, ps);
        std::vector<float> image((size_t)model->size());
        aio_ops::ck(aio_tomo_ext_adjoint_wavefield(context(0), image.data(), 0, _reflectivityExt->getVals(), &sh,
                                                   AIO_MEM_HOST, _wSrc->getVals(), _wSec1->getVals(),
                                                   _wSec2->getVals()));
    }
    std::shared_ptr<SEP::float3DReg> getSrcWavefield() { return _wSrc; }
    std::shared_ptr<SEP::float3DReg> getSecWavefield1() { return _wSec1; }
    std::shared_ptr<SEP::float3DReg> getSecWavefield2() { return _wSec2; }
    void setVel(std::shared_ptr<SEP::float2DReg> vel) { setVelocity(vel); }
    void setReflectivityExt(std::shared_ptr<SEP::float3DReg> reflectivityExt) { _reflectivityExt = reflectivityExt; }

  private:
    std::shared_ptr<SEP::float3DReg> _reflectivityExt;
};

// Extended WEMVA: velocity perturbation [nx][nz] -> extended image [nExt][nx][nz], with the
// observed data of every shot driving the receiver wavefield (F/src/wemvaExtShotsGpu.cpp).
class wemvaExtShotsGpu : public Operator<SEP::float2DReg, SEP::float3DReg>, public aio_ops::BornFamily<SEP::float2DReg> {
  public:
    // the dot-product test reduces on the first GPU of the operator's list
    int dotTestDevice() const override { return _gpuList.empty() || _gpuList[0] < 0 ? 0 : _gpuList[0]; }
    wemvaExtShotsGpu(std::shared_ptr<SEP::float2DReg> vel, std::shared_ptr<paramObj> par,
                     std::vector<std::shared_ptr<deviceGpu>> sourcesVector,
                     std::vector<std::shared_ptr<SEP::float2DReg>> sourcesSignalsVector,
                     std::vector<std::shared_ptr<deviceGpu>> receiversVector,
                     std::vector<std::shared_ptr<SEP::float2DReg>> receiversSignalsVector)
        : BornFamily(vel, par, AIO_WEMVA_EXT, sourcesVector, sourcesSignalsVector, receiversVector) {
        _receiversSignalsVector = receiversSignalsVector;
        _freeSurfaceDrivers = false;
    }

    void forward(const bool add, const std::shared_ptr<SEP::float2DReg> model,
                 std::shared_ptr<SEP::float3DReg> data) const override {
        std::vector<std::vector<float>> parts(_nGpu);
        const size_t n = (size_t)data->size();
        forShots(nullptr, true, [&](int g, int, int, std::vector<aio_ops::PreparedShot>&, std::vector<aio_shot>& sh) {
            parts[g].assign(n, 0.f);
            aio_ops::ck(aio_wemva_ext_forward(context(g), model->getVals(), parts[g].data(), 0, (int)sh.size(), sh.data(),
                                              AIO_MEM_HOST));
        });
        sumImages(parts, data->getVals(), n, add);
    }
    void adjoint(const bool add, std::shared_ptr<SEP::float2DReg> model,
                 const std::shared_ptr<SEP::float3DReg> data) const override {
        std::vector<std::vector<float>> parts(_nGpu);
        const size_t n = (size_t)model->size();
        forShots(nullptr, true, [&](int g, int, int, std::vector<aio_ops::PreparedShot>&, std::vector<aio_shot>& sh) {
            parts[g].assign(n, 0.f);
            aio_ops::ck(aio_wemva_ext_adjoint(context(g), parts[g].data(), 0, data->getVals(), (int)sh.size(), sh.data(),
                                              AIO_MEM_HOST));
        });
        sumImages(parts, model->getVals(), n, add);
    }
    // forward / adjoint of every shot, plus, with saveWavefield = 1, the saved wavefields of shot
    // wavefieldShotNumber (F/src/wemvaExtShotsGpu.cpp forwardWavefield / adjointWavefield): d2/dt2
    // of the source wavefield, the receiver wavefield and the last leg's scattered samples. With
    // saveWavefield = 0 the containers stay zero-filled.
    void forwardWavefield(const bool add, const std::shared_ptr<SEP::float2DReg> model,
                          std::shared_ptr<SEP::float3DReg> data) {
        forward(add, model, data);
        resetWavefields3();
        if (!wavefieldShotValid()) return;
        aio_ops::PreparedShot ps;
        aio_shot sh = prepareOne(_wavefieldShotNumber, nullptr, ps, true);
        std::vector<float> image((size_t)data->size());
        aio_ops::ck(aio_wemva_ext_forward_wavefield(context(0), model->getVals(), image.data(), 0, &sh, AIO_MEM_HOST,
                                                    _wSrc->getVals(), _wSec1->getVals(), _wSec2->getVals()));
    }
    void adjointWavefield(const bool add, std::shared_ptr<SEP::float2DReg> model,
                          const std::shared_ptr<SEP::float3DReg> data) {
        adjoint(add, model, data);
        resetWavefields3();
        if (!wavefieldShotValid()) return;
        aio_ops::PreparedShot ps;
        aio_shot sh = prepareOne(_wavefieldShotNumber, nullptr, ps, true);
        std::vector<float> m((size_t)model->size());
        aio_ops::ck(aio_wemva_ext_adjoint_wavefield(context(0), m.data(), 0, data->getVals(), &sh, AIO_MEM_HOST,
                                                    _wSrc->getVals(), _wSec1->getVals(), _wSec2->getVals()));
    }
    std::shared_ptr<SEP::float3DReg> getSrcWavefield() { return _wSrc; }
    std::shared_ptr<SEP::float3DReg> getSecWavefield1() { return _wSec1; }
    std::shared_ptr<SEP::float3DReg> getSecWavefield2() { return _wSec2; }
    void setVel(std::shared_ptr<SEP::float2DReg> vel) { setVelocity(vel); }
    void setReceiversSignalsVector(std::vector<std::shared_ptr<SEP::float2DReg>> v) { _receiversSignalsVector = v; }
};
