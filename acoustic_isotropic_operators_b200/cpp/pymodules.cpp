// pybind11 modules with the reference's module and class names
// (P/python_float/pyAcoustic_iso_float_{nl,born,born_ext,tomo,wemva}.cpp) over the
// B200 operator classes, plus pySepLite for the SEP-compatible containers and
// parameter dictionaries those classes take. One source, compiled once per
// module with AIO_MODULE set to 0 (pySepLite), 1 (nl), 2 (born), 3 (born_ext),
// 4 (tomo) or 5 (wemva).
#include <pybind11/iostream.h>
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include "aio_sepio.hpp"
#include "aio_shots.hpp"

namespace py = pybind11;

#if AIO_MODULE == 0
template <class V>
static void bind_vector(py::module_& m, const char* name) {
    py::class_<V, std::shared_ptr<V>>(m, name)
        .def(py::init<std::shared_ptr<SEP::hypercube>>())
        .def("getHyper", &V::getHyper)
        .def("getNdArray",
             [](V& v) {
                 // numpy view, slowest axis first (reference getNdArray convention)
                 std::vector<py::ssize_t> shape;
                 auto h = v.getHyper();
                 for (int i = h->getNdim(); i >= 1; i--) shape.push_back(h->getAxis(i).n);
                 std::vector<py::ssize_t> strides(shape.size());
                 py::ssize_t s = sizeof(float);
                 for (int i = (int)shape.size() - 1; i >= 0; i--) {
                     strides[i] = s;
                     s *= shape[i];
                 }
                 return py::array_t<float>(shape, strides, v.getVals(), py::cast(&v));
             })
        .def("scale", &V::scale)
        .def("set", &V::set)
        .def("zero", &V::zero)
        .def("random", &V::random)
        .def("clone", [](const V& v) { return v.clone(); })
        .def("cloneSpace", [](const V& v) { return v.cloneSpace(); })
        .def("dot", [](const V& v, std::shared_ptr<V> o) { return v.dot(o); })
        .def("scaleAdd", [](V& v, std::shared_ptr<V> o, double a, double b) { v.scaleAdd(o, a, b); })
        .def("checkSame", [](const V& v, std::shared_ptr<V> o) { return v.checkSame(o); })
        .def("max", &V::max)
        .def("min", &V::min);
}

PYBIND11_MODULE(pySepLite, m) {
    m.doc() = "SEP-compatible containers (axis, hypercube, float1/2/3DReg, paramObj) for the operator modules";
    py::class_<SEP::axis>(m, "axis")
        .def(py::init<int, float, float, const std::string&, const std::string&>(), py::arg("n"), py::arg("o") = 0.f,
             py::arg("d") = 1.f, py::arg("label") = "", py::arg("unit") = "")
        .def_readwrite("n", &SEP::axis::n)
        .def_readwrite("o", &SEP::axis::o)
        .def_readwrite("d", &SEP::axis::d);
    py::class_<SEP::hypercube, std::shared_ptr<SEP::hypercube>>(m, "hypercube")
        .def(py::init<const std::vector<SEP::axis>&>())
        .def("getAxis", &SEP::hypercube::getAxis)
        .def("getNdim", &SEP::hypercube::getNdim)
        .def("getN123", &SEP::hypercube::getN123)
        .def("getNs", &SEP::hypercube::getNs);
    bind_vector<SEP::float1DReg>(m, "float1DReg");
    bind_vector<SEP::float2DReg>(m, "float2DReg");
    bind_vector<SEP::float3DReg>(m, "float3DReg");
    py::class_<paramObj, std::shared_ptr<paramObj>>(m, "paramObj")
        .def("getInt", py::overload_cast<const std::string&, int>(&paramObj::getInt, py::const_))
        .def("getFloat", py::overload_cast<const std::string&, float>(&paramObj::getFloat, py::const_))
        .def("getString", py::overload_cast<const std::string&, const std::string&>(&paramObj::getString, py::const_));
    py::class_<dictParams, paramObj, std::shared_ptr<dictParams>>(m, "dictParams")
        .def(py::init([](py::dict d) {
            auto p = std::make_shared<dictParams>();
            for (auto kv : d) {
                std::string v;
                if (py::isinstance<py::list>(kv.second) || py::isinstance<py::tuple>(kv.second)) {
                    for (auto e : kv.second) v += (v.empty() ? "" : ",") + py::str(e).cast<std::string>();
                } else {
                    v = py::str(kv.second).cast<std::string>();
                }
                p->set(py::str(kv.first).cast<std::string>(), v);
            }
            return p;
        }))
        .def("set", &dictParams::set);
    py::class_<SEP::argParams, paramObj, std::shared_ptr<SEP::argParams>>(m, "argParams")
        .def(py::init<const std::vector<std::string>&>(), "parameters from key=value arguments and par= files")
        .def("getInts", py::overload_cast<const std::string&>(&paramObj::getInts, py::const_));
    // SEP .H datasets (genericIO.defaultIO.getVector / writeVector of the reference's Python)
    m.def(
        "getVector",
        [](const std::string& path, int ndims) -> py::object {
            SEP::genericRegFile f(path, usageIn);
            auto h = f.getHyper();
            if (ndims <= 0) ndims = h->getNdim();
            if (ndims < h->getNdim() || ndims > 3)
                throw std::runtime_error("SEP: " + path + " has " + std::to_string(h->getNdim()) +
                                         " axes; vectors of 1 to 3 axes, at least as many as the file's");
            while (h->getNdim() < ndims) h->addAxis(SEP::axis(1));
            auto read = [&](auto v) -> py::object {
                f.readFloatStream(v);
                return py::cast(v);
            };
            if (ndims == 1) return read(std::make_shared<SEP::float1DReg>(h));
            if (ndims == 2) return read(std::make_shared<SEP::float2DReg>(h));
            return read(std::make_shared<SEP::float3DReg>(h));
        },
        py::arg("path"), py::arg("ndims") = 0);
    m.def("writeVector", [](const std::string& p, std::shared_ptr<SEP::float1DReg> v, const std::string& f) {
        SEP::writeVector(p, v, f);
    }, py::arg("path"), py::arg("vec"), py::arg("data_format") = "xdr_float");
    m.def("writeVector", [](const std::string& p, std::shared_ptr<SEP::float2DReg> v, const std::string& f) {
        SEP::writeVector(p, v, f);
    }, py::arg("path"), py::arg("vec"), py::arg("data_format") = "xdr_float");
    m.def("writeVector", [](const std::string& p, std::shared_ptr<SEP::float3DReg> v, const std::string& f) {
        SEP::writeVector(p, v, f);
    }, py::arg("path"), py::arg("vec"), py::arg("data_format") = "xdr_float");
}

#elif AIO_MODULE == 1
PYBIND11_MODULE(pyAcoustic_iso_float_nl, m) {
    py::module_::import("pySepLite");
    py::add_ostream_redirect(m, "ostream_redirect");
    py::class_<deviceGpu, std::shared_ptr<deviceGpu>>(m, "deviceGpu")
        .def(py::init<const std::shared_ptr<SEP::float1DReg>, const std::shared_ptr<SEP::float1DReg>,
                      const std::shared_ptr<SEP::float2DReg>, int&, int, float, float>(),
             "Initialize a deviceGpu object using location, velocity, and nt")
        .def(py::init<const std::vector<int>&, const std::vector<int>&, const std::shared_ptr<SEP::float2DReg>, int&,
                      int, int, int>(),
             "Initialize a deviceGpu object using coordinates and nt")
        .def(py::init<const int&, const int&, const int&, const int&, const int&, const int&,
                      const std::shared_ptr<SEP::float2DReg>, int&, int, int, int>(),
             "Initialize a deviceGpu object using sampling in z and x axes, velocity, and nt")
        .def("forward", &deviceGpu::forward, "regular [nDeviceReg][nt] -> devices [nDeviceIrreg][nt]")
        .def("adjoint", &deviceGpu::adjoint, "devices -> regular")
        .def("setDomainRange", &deviceGpu::setDomainRange)
        .def("dotTest", &deviceGpu::dotTest, py::arg("verbose") = false, py::arg("maxError") = 1e-5f)
        .def("getNDeviceReg", &deviceGpu::getNDeviceReg)
        .def("getNDeviceIrreg", &deviceGpu::getNDeviceIrreg)
        .def("getRegPosUnique", [](deviceGpu& d) {
            return std::vector<int>(d.getRegPosUnique(), d.getRegPosUnique() + d.getNDeviceReg());
        })
        .def("getRegPos", [](deviceGpu& d) {  // corner grid indices, nCorner per device
            return std::vector<int>(d.getRegPos(), d.getRegPos() + d.nCorner() * d.getNDeviceIrreg());
        })
        .def("getWeights", [](deviceGpu& d) {  // corner weights, same order as getRegPos
            return std::vector<float>(d.getWeights(), d.getWeights() + d.nCorner() * d.getNDeviceIrreg());
        })
        .def("getNt", &deviceGpu::getNt)
        .def_static("windowedSinc", &deviceGpu::windowedSinc, "Kaiser-windowed sinc devices at coordinates",
                    py::arg("zCoord"), py::arg("xCoord"), py::arg("vel"), py::arg("nt"), py::arg("halfWidth") = 4,
                    py::arg("beta") = 4.14f, py::arg("dipole") = 0, py::arg("zDipoleShift") = 0.f,
                    py::arg("xDipoleShift") = 0.f);
    py::class_<nonlinearPropShotsGpu, std::shared_ptr<nonlinearPropShotsGpu>>(m, "nonlinearPropShotsGpu")
        .def(py::init<std::shared_ptr<SEP::float2DReg>, std::shared_ptr<paramObj>, std::vector<std::shared_ptr<deviceGpu>>,
                      std::vector<std::shared_ptr<deviceGpu>>>(),
             "Initialize a nonlinearPropShotsGpu")
        .def("forward", &nonlinearPropShotsGpu::forward, "Forward")
        .def("setDomainRange", &nonlinearPropShotsGpu::setDomainRange, "Domain and range vectors (used by dotTest)")
        .def("adjoint", &nonlinearPropShotsGpu::adjoint, "Adjoint")
        .def("forwardWavefield", &nonlinearPropShotsGpu::forwardWavefield, "Forward wavefield")
        .def("adjointWavefield", &nonlinearPropShotsGpu::adjointWavefield, "Adjoint wavefield")
        .def("setVel", &nonlinearPropShotsGpu::setVel, "Function to set background velocity")
        .def("dotTest", &nonlinearPropShotsGpu::dotTest, "Dot-Product Test", py::arg("verbose") = false,
             py::arg("maxError") = 1e-5f)
        .def("getWfld", &nonlinearPropShotsGpu::getWavefield, "Function to get nl wavefield");
}

#elif AIO_MODULE == 2
PYBIND11_MODULE(pyAcoustic_iso_float_born, m) {
    py::module_::import("pyAcoustic_iso_float_nl");
    py::add_ostream_redirect(m, "ostream_redirect");
    py::class_<BornShotsGpu, std::shared_ptr<BornShotsGpu>>(m, "BornShotsGpu")
        .def(py::init<std::shared_ptr<SEP::float2DReg>, std::shared_ptr<paramObj>, std::vector<std::shared_ptr<deviceGpu>>,
                      std::vector<std::shared_ptr<SEP::float2DReg>>, std::vector<std::shared_ptr<deviceGpu>>>(),
             "Initialize a BornShotsGpu")
        .def("forward", &BornShotsGpu::forward, "Forward")
        .def("setDomainRange", &BornShotsGpu::setDomainRange, "Domain and range vectors (used by dotTest)")
        .def("adjoint", &BornShotsGpu::adjoint, "Adjoint")
        .def("forwardWavefield", &BornShotsGpu::forwardWavefield, "Forward wavefield")
        .def("adjointWavefield", &BornShotsGpu::adjointWavefield, "Adjoint wavefield")
        .def("setVel", &BornShotsGpu::setVel, "Function to set background velocity")
        .def("dotTest", &BornShotsGpu::dotTest, "Dot-Product Test", py::arg("verbose") = false, py::arg("maxError") = 1e-5f)
        .def("getSrcWfld", &BornShotsGpu::getSrcWavefield, "Function to get src wfld")
        .def("getSecWfld", &BornShotsGpu::getSecWavefield, "Function to get adj wfld");
}

#elif AIO_MODULE == 3
PYBIND11_MODULE(pyAcoustic_iso_float_born_ext, m) {
    py::module_::import("pyAcoustic_iso_float_nl");
    py::add_ostream_redirect(m, "ostream_redirect");
    py::class_<BornExtShotsGpu, std::shared_ptr<BornExtShotsGpu>>(m, "BornExtShotsGpu")
        .def(py::init<std::shared_ptr<SEP::float2DReg>, std::shared_ptr<paramObj>, std::vector<std::shared_ptr<deviceGpu>>,
                      std::vector<std::shared_ptr<SEP::float2DReg>>, std::vector<std::shared_ptr<deviceGpu>>>(),
             "Initialize a BornExtShotsGpu")
        .def("forward", &BornExtShotsGpu::forward, "Forward")
        .def("setDomainRange", &BornExtShotsGpu::setDomainRange, "Domain and range vectors (used by dotTest)")
        .def("adjoint", &BornExtShotsGpu::adjoint, "Adjoint")
        .def("forwardWavefield", &BornExtShotsGpu::forwardWavefield, "Forward wavefield")
        .def("adjointWavefield", &BornExtShotsGpu::adjointWavefield, "Adjoint wavefield")
        .def("setVel", &BornExtShotsGpu::setVel, "Function to set background velocity")
        .def("getVel", &BornExtShotsGpu::getVel, "Function to get background velocity")
        .def("getSrcWfld", &BornExtShotsGpu::getSrcWavefield, "Function to get src wfld")
        .def("getSecWfld", &BornExtShotsGpu::getSecWavefield, "Function to get scattered / receiver wfld")
        .def("dotTest", &BornExtShotsGpu::dotTest, "Dot-Product Test", py::arg("verbose") = false,
             py::arg("maxError") = 1e-5f);
}

#elif AIO_MODULE == 4
PYBIND11_MODULE(pyAcoustic_iso_float_tomo, m) {
    py::module_::import("pyAcoustic_iso_float_nl");
    py::add_ostream_redirect(m, "ostream_redirect");
    py::class_<tomoExtShotsGpu, std::shared_ptr<tomoExtShotsGpu>>(m, "tomoExtShotsGpu")
        .def(py::init<std::shared_ptr<SEP::float2DReg>, std::shared_ptr<paramObj>, std::vector<std::shared_ptr<deviceGpu>>,
                      std::vector<std::shared_ptr<SEP::float2DReg>>, std::vector<std::shared_ptr<deviceGpu>>,
                      std::shared_ptr<SEP::float3DReg>>(),
             "Initialize a tomoExtShotsGpu")
        .def("forward", &tomoExtShotsGpu::forward, "Forward")
        .def("setDomainRange", &tomoExtShotsGpu::setDomainRange, "Domain and range vectors (used by dotTest)")
        .def("adjoint", &tomoExtShotsGpu::adjoint, "Adjoint")
        .def("forwardWavefield", &tomoExtShotsGpu::forwardWavefield, "Forward wavefield")
        .def("adjointWavefield", &tomoExtShotsGpu::adjointWavefield, "Adjoint wavefield")
        .def("getSrcWavefield", &tomoExtShotsGpu::getSrcWavefield, "Saved d2/dt2 of the source wavefield")
        .def("getSecWavefield1", &tomoExtShotsGpu::getSecWavefield1, "First saved secondary wavefield")
        .def("getSecWavefield2", &tomoExtShotsGpu::getSecWavefield2, "Second saved secondary wavefield")
        .def("setVel", &tomoExtShotsGpu::setVel, "Function to set background velocity")
        .def("setReflectivityExt", &tomoExtShotsGpu::setReflectivityExt, "Function to set reflectivity")
        .def("dotTest", &tomoExtShotsGpu::dotTest, "Dot-Product Test", py::arg("verbose") = false,
             py::arg("maxError") = 1e-5f);
}

#elif AIO_MODULE == 5
PYBIND11_MODULE(pyAcoustic_iso_float_wemva, m) {
    py::module_::import("pyAcoustic_iso_float_nl");
    py::add_ostream_redirect(m, "ostream_redirect");
    py::class_<wemvaExtShotsGpu, std::shared_ptr<wemvaExtShotsGpu>>(m, "wemvaExtShotsGpu")
        .def(py::init<std::shared_ptr<SEP::float2DReg>, std::shared_ptr<paramObj>, std::vector<std::shared_ptr<deviceGpu>>,
                      std::vector<std::shared_ptr<SEP::float2DReg>>, std::vector<std::shared_ptr<deviceGpu>>,
                      std::vector<std::shared_ptr<SEP::float2DReg>>>(),
             "Initialize a wemvaExtShotsGpu")
        .def("forward", &wemvaExtShotsGpu::forward, "Forward")
        .def("setDomainRange", &wemvaExtShotsGpu::setDomainRange, "Domain and range vectors (used by dotTest)")
        .def("adjoint", &wemvaExtShotsGpu::adjoint, "Adjoint")
        .def("forwardWavefield", &wemvaExtShotsGpu::forwardWavefield, "Forward wavefield")
        .def("adjointWavefield", &wemvaExtShotsGpu::adjointWavefield, "Adjoint wavefield")
        .def("getSrcWavefield", &wemvaExtShotsGpu::getSrcWavefield, "Saved d2/dt2 of the source wavefield")
        .def("getSecWavefield1", &wemvaExtShotsGpu::getSecWavefield1, "First saved secondary wavefield")
        .def("getSecWavefield2", &wemvaExtShotsGpu::getSecWavefield2, "Second saved secondary wavefield")
        .def("setVel", &wemvaExtShotsGpu::setVel, "Function to set background velocity")
        .def("setReceiversSignalsVector", &wemvaExtShotsGpu::setReceiversSignalsVector, "Set the WEMVA data")
        .def("dotTest", &wemvaExtShotsGpu::dotTest, "Dot-Product Test", py::arg("verbose") = false,
             py::arg("maxError") = 1e-5f);
}
#endif
