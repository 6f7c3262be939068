// Fortran formatted output (the edit descriptors the reference's text files
// use), for the host-side file writers.  A record is built item by item; an
// X edit descriptor after the last item transmits nothing (it does not extend
// the record), so separators are written only between items.
#pragma once
#include <cstdio>
#include <string>

namespace dmfted {
namespace fort {

// Aw: right-justified in w characters; a longer string keeps its first w.
inline std::string A(const std::string &s, int w) {
    if ((int)s.size() >= w) return s.substr(0, w);
    return std::string(w - s.size(), ' ') + s;
}

// Fw.d of a finite value; a field too narrow is all '*'.
inline std::string F(double x, int w, int d) {
    char buf[64];
    std::snprintf(buf, sizeof buf, "%*.*f", w, d, x);
    std::string s(buf);
    if ((int)s.size() > w) return std::string(w, '*');
    return s;
}

// ESw.d: one digit before the point, d after, exponent "E+dd"; a three-digit
// exponent drops the letter ("+ddd"), the standard's form for |exp| > 99
// with no Ee given.
inline std::string ES(double x, int w, int d) {
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.*E", d, x);
    std::string s(buf);
    const size_t e = s.find('E');
    if (e != std::string::npos) {
        const std::string mant = s.substr(0, e);
        const char sign = s[e + 1];
        std::string digs = s.substr(e + 2);
        while (digs.size() > 2 && digs[0] == '0') digs.erase(0, 1);
        if (digs.size() <= 2) {
            if (digs.size() < 2) digs = "0" + digs;
            s = mant + "E" + sign + digs;
        } else {
            s = mant + sign + digs;
        }
    }
    if ((int)s.size() > w) return std::string(w, '*');
    return std::string(w - s.size(), ' ') + s;
}

// Iw.
inline std::string I(long long v, int w) {
    char buf[64];
    std::snprintf(buf, sizeof buf, "%*lld", w, v);
    std::string s(buf);
    if ((int)s.size() > w) return std::string(w, '*');
    return s;
}

// A record of items with `sep` between them ("(90(F15.9,1X))": sep " ").
struct Record {
    std::string s;
    std::string sep;
    bool first = true;
    explicit Record(std::string separator = " ") : sep(std::move(separator)) {}
    Record &add(const std::string &item) {
        if (!first) s += sep;
        s += item;
        first = false;
        return *this;
    }
};

}  // namespace fort
}  // namespace dmfted
