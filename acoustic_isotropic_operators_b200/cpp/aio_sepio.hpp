// SEP file I/O for the operator layer: .H headers with a separate binary data file,
// parameters from the command line and par files, and the genericIO calls the
// reference's programs make on them (F/src/BornShotsGpuMain.cpp:24-25,87-90,158-160,
// 199-234: getDefaultIO, getParamObj, getRegFile(tag, usage), getHyper / setHyper,
// readFloatStream, writeDescription, writeFloatStream).
//
// Header format (SEP): text of key=value tokens, later tokens overriding earlier ones,
// values optionally in double or single quotes. Keys read: n1..n9, o1..o9, d1..d9,
// label1..9, unit1..9, in (path of the data file), esize (4: float samples) and
// data_format ("xdr_float", big-endian, the default when absent; or "native_float",
// the host's byte order). The number of dimensions of a read hypercube is that of its
// last axis longer than 1 (at least 1), as SEP's readers report it. Written headers
// name the data file `<header path>@`, or `$DATAPATH<header file name>@` when the
// DATAPATH environment variable is set.
#pragma once
#include <algorithm>
#include <cctype>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>

#include "aio_sep.hpp"

enum usage_t { usageIn, usageOut, usageInOut, usageScr };

namespace SEP {

// key=value tokens of a header or par file, in order (later ones override earlier ones)
inline std::vector<std::pair<std::string, std::string>> sepTokens(const std::string& text, bool comments) {
    std::vector<std::pair<std::string, std::string>> out;
    const size_t n = text.size();
    size_t i = 0;
    auto keyChar = [](char c) { return std::isalnum((unsigned char)c) || c == '_' || c == '.'; };
    while (i < n) {
        if (comments && text[i] == '#') {
            while (i < n && text[i] != '\n') i++;
            continue;
        }
        if (text[i] != '=') {
            i++;
            continue;
        }
        size_t k = i;
        while (k > 0 && keyChar(text[k - 1])) k--;
        const std::string key = text.substr(k, i - k);
        size_t j = i + 1;
        std::string val;
        if (j < n && (text[j] == '"' || text[j] == '\'')) {
            const char q = text[j];
            const size_t e = text.find(q, j + 1);
            if (e == std::string::npos) throw std::runtime_error("SEP: unterminated quote after " + key + "=");
            val = text.substr(j + 1, e - j - 1);
            j = e + 1;
        } else {
            size_t e = j;
            while (e < n && !std::isspace((unsigned char)text[e])) e++;
            val = text.substr(j, e - j);
            j = e;
        }
        if (!key.empty()) out.emplace_back(key, val);
        i = j;
    }
    return out;
}

inline std::string sepReadText(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("SEP: cannot open " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    return ss.str();
}

// paramObj over command-line arguments key=value; par=<file> inserts the file's tokens at
// its place ('#' starts a comment there). Later occurrences override earlier ones.
class argParams : public paramObj {
  public:
    argParams() = default;
    argParams(int argc, char** argv) {
        std::vector<std::string> a;
        for (int i = 1; i < argc; i++) a.emplace_back(argv[i]);
        add(a);
    }
    explicit argParams(const std::vector<std::string>& args) { add(args); }
    bool has(const std::string& k) const override { return _m.count(k) > 0; }
    std::string raw(const std::string& k) const override { return _m.at(k); }

  private:
    void add(const std::vector<std::string>& args) {
        for (const auto& s : args) {
            for (const auto& kv : sepTokens(s, false)) {
                if (kv.first == "par") addFile(kv.second, 0);
                else _m[kv.first] = kv.second;
            }
        }
    }
    void addFile(const std::string& path, int depth) {
        if (depth > 8) throw std::runtime_error("SEP: par files nested too deep at " + path);
        for (const auto& kv : sepTokens(sepReadText(path), true)) {
            if (kv.first == "par") addFile(kv.second, depth + 1);
            else _m[kv.first] = kv.second;
        }
    }
    std::map<std::string, std::string> _m;
};

// One SEP dataset: header + binary data file, read or written as a stream of floats.
class genericRegFile {
  public:
    genericRegFile(const std::string& header, usage_t usage) : _header(header), _usage(usage) {
        if (usage == usageIn || usage == usageInOut) parse();
    }
    ~genericRegFile() {
        if (_data) std::fclose(_data);
    }
    genericRegFile(const genericRegFile&) = delete;
    genericRegFile& operator=(const genericRegFile&) = delete;

    std::shared_ptr<hypercube> getHyper() const {
        if (!_hyper) throw std::runtime_error("SEP: " + _header + " has no hypercube yet");
        return std::make_shared<hypercube>(*_hyper);
    }
    void setHyper(std::shared_ptr<hypercube> h) { _hyper = std::make_shared<hypercube>(*h); }
    void setDataFormat(const std::string& f) {
        if (f != "xdr_float" && f != "native_float") throw std::runtime_error("SEP: unsupported data_format " + f);
        _format = f;
    }
    std::string getDataFormat() const { return _format; }
    std::string getDataPath() const { return _dataPath; }
    // header keys of a read file (n1, o1, in, data_format, ...)
    bool hasKey(const std::string& k) const { return _keys.count(k) > 0; }
    std::string getKey(const std::string& k) const { return _keys.at(k); }

    // Writes the header (hypercube, esize, data_format, in) and starts an empty data file.
    void writeDescription() {
        if (!_hyper) throw std::runtime_error("SEP: setHyper before writeDescription on " + _header);
        _dataPath = dataPathFor(_header);
        std::ofstream h(_header);
        if (!h) throw std::runtime_error("SEP: cannot write " + _header);
        h << "\naio_sepio: SEP dataset written by the operator layer\n";
        for (int i = 1; i <= _hyper->getNdim(); i++) {
            const axis a = _hyper->getAxis(i);
            h << "\t\tn" << i << "=" << a.n << " o" << i << "=" << fmt(a.o) << " d" << i << "=" << fmt(a.d);
            if (!a.label.empty()) h << " label" << i << "=\"" << a.label << "\"";
            if (!a.unit.empty()) h << " unit" << i << "=\"" << a.unit << "\"";
            h << "\n";
        }
        h << "\t\tesize=4\n\t\tdata_format=\"" << _format << "\"\n\t\tin=\"" << _dataPath << "\"\n";
        if (!h) throw std::runtime_error("SEP: cannot write " + _header);
        if (_data) std::fclose(_data);
        _data = std::fopen(_dataPath.c_str(), "wb");
        if (!_data) throw std::runtime_error("SEP: cannot create " + _dataPath);
    }
    void writeFloatStream(const float* p, long long n) {
        if (!_data || _usage == usageIn) throw std::runtime_error("SEP: writeDescription before writing " + _header);
        const long long chunk = 1 << 20;  // byte-swapped through a bounded buffer
        std::vector<float> buf((size_t)std::min(n, chunk));
        for (long long o = 0; o < n; o += chunk) {
            const long long m = std::min(chunk, n - o);
            std::copy(p + o, p + o + m, buf.begin());
            if (swap()) swapBytes(buf.data(), m);
            if (std::fwrite(buf.data(), 4, (size_t)m, _data) != (size_t)m)
                throw std::runtime_error("SEP: short write to " + _dataPath);
        }
        std::fflush(_data);
    }
    template <class V>
    void writeFloatStream(const std::shared_ptr<V> v) {
        writeFloatStream(v->getVals(), v->size());
    }
    void readFloatStream(float* p, long long n) {
        if (!_data) {
            _data = std::fopen(_dataPath.c_str(), "rb");
            if (!_data) throw std::runtime_error("SEP: cannot open data file " + _dataPath);
        }
        if (std::fread(p, 4, (size_t)n, _data) != (size_t)n)
            throw std::runtime_error("SEP: " + _dataPath + " holds fewer samples than requested");
        if (swap()) swapBytes(p, n);
    }
    template <class V>
    void readFloatStream(std::shared_ptr<V> v) {
        readFloatStream(v->getVals(), v->size());
    }

  private:
    void parse() {
        for (const auto& kv : sepTokens(sepReadText(_header), false)) _keys[kv.first] = kv.second;
        std::vector<axis> ax;
        int last = 1;
        for (int i = 1; i <= 9; i++) {
            const std::string s = std::to_string(i);
            axis a(1);
            if (_keys.count("n" + s)) a.n = std::stoi(_keys["n" + s]);
            if (_keys.count("o" + s)) a.o = std::stof(_keys["o" + s]);
            if (_keys.count("d" + s)) a.d = std::stof(_keys["d" + s]);
            if (_keys.count("label" + s)) a.label = _keys["label" + s];
            if (_keys.count("unit" + s)) a.unit = _keys["unit" + s];
            if (a.n < 1) throw std::runtime_error("SEP: n" + s + " < 1 in " + _header);
            if (a.n > 1) last = i;
            ax.push_back(a);
        }
        ax.resize(last);
        _hyper = std::make_shared<hypercube>(ax);
        if (_keys.count("esize") && std::stoi(_keys["esize"]) != 4)
            throw std::runtime_error("SEP: only esize=4 (float) datasets are supported: " + _header);
        if (_keys.count("data_format")) setDataFormat(_keys["data_format"]);
        if (!_keys.count("in") || _keys["in"] == "stdin" || _keys["in"] == "-1")
            throw std::runtime_error("SEP: " + _header + " names no separate data file (in=)");
        _dataPath = _keys["in"];
    }
    static std::string dataPathFor(const std::string& header) {
        const char* dp = std::getenv("DATAPATH");
        if (!dp || !*dp) return header + "@";
        const size_t slash = header.find_last_of('/');
        return std::string(dp) + (slash == std::string::npos ? header : header.substr(slash + 1)) + "@";
    }
    static std::string fmt(float v) {
        std::ostringstream s;
        s.precision(9);
        s << v;
        return s.str();
    }
    bool swap() const {
        const uint32_t one = 1;
        unsigned char b;
        std::memcpy(&b, &one, 1);
        const bool little = b == 1;
        return _format == "xdr_float" ? little : false;
    }
    static void swapBytes(float* p, long long n) {
        for (long long i = 0; i < n; i++) {
            uint32_t u;
            std::memcpy(&u, p + i, 4);
            u = (u >> 24) | ((u >> 8) & 0xff00u) | ((u << 8) & 0xff0000u) | (u << 24);
            std::memcpy(p + i, &u, 4);
        }
    }

    std::string _header, _dataPath, _format = "xdr_float";
    usage_t _usage;
    std::map<std::string, std::string> _keys;
    std::shared_ptr<hypercube> _hyper;
    std::FILE* _data = nullptr;
};

// genericIO over SEP files: parameters from the command line, datasets by tag (the value
// of parameter `tag` when it is given, else `tag` itself as the header path).
class genericIO {
  public:
    explicit genericIO(std::shared_ptr<paramObj> par) : _par(std::move(par)) {}
    std::shared_ptr<paramObj> getParamObj() const { return _par; }
    std::shared_ptr<genericRegFile> getRegFile(const std::string& tag, usage_t usage) const {
        const std::string path = _par && _par->has(tag) ? _par->raw(tag) : tag;
        return std::make_shared<genericRegFile>(path, usage);
    }

  private:
    std::shared_ptr<paramObj> _par;
};

class ioModes {
  public:
    ioModes(int argc, char** argv) : _io(std::make_shared<genericIO>(std::make_shared<argParams>(argc, argv))) {}
    std::shared_ptr<genericIO> getDefaultIO() const { return _io; }

  private:
    std::shared_ptr<genericIO> _io;
};

// Whole-dataset helpers (genericIO.defaultIO.getVector / writeVector in the reference's Python)
template <class V>
std::shared_ptr<V> readVector(const std::string& header) {
    genericRegFile f(header, usageIn);
    auto v = std::make_shared<V>(f.getHyper());
    f.readFloatStream(v);
    return v;
}
template <class V>
void writeVector(const std::string& header, const std::shared_ptr<V> v, const std::string& format = "xdr_float") {
    genericRegFile f(header, usageOut);
    f.setHyper(v->getHyper());
    f.setDataFormat(format);
    f.writeDescription();
    f.writeFloatStream(v);
}

}  // namespace SEP
