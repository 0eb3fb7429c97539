// or_deck.hpp -- Fortran list-directed record reader for the oracle's deck parser.
//
// TEST INFRASTRUCTURE ONLY (see evp_oracle.h).  Restates the record semantics
// the reference's READ statements rely on (IO_functions.f90:51-346):
//   read(u,*) a,b,c   -> values from the next record(s); the rest of the last
//                        record used is skipped; blanks, tabs and commas
//                        separate; '/' ends the list; Fortran 'd' exponents.
//   read(u,*)         -> skip one record
//   read(u,'(a)') s   -> the whole next record
#pragma once
#include <string>
#include <vector>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <cstdlib>

namespace orc {

struct DeckError : std::runtime_error {
    explicit DeckError(const std::string& m) : std::runtime_error(m) {}
};

class RecordReader {
public:
    RecordReader() {}
    explicit RecordReader(const std::string& path) { open(path); }
    void open(const std::string& path) {
        std::ifstream f(path);
        if (!f) throw DeckError("cannot open file '" + path + "'");
        path_ = path;
        std::string line;
        while (std::getline(f, line)) {
            if (!line.empty() && line.back() == '\r') line.pop_back();
            lines_.push_back(line);
        }
        pos_ = 0;
    }
    std::string read_line() {
        if (pos_ >= lines_.size()) throw DeckError("unexpected end of file in '" + path_ + "'");
        return lines_[pos_++];
    }
    void skip() { read_line(); }
    // Read n list-directed tokens (numbers stay as text).
    std::vector<std::string> read_tokens(size_t n) {
        std::vector<std::string> out;
        while (out.size() < n) {
            std::string rec = read_line();
            size_t i = 0;
            bool slash = false;
            while (i < rec.size() && out.size() < n) {
                char c = rec[i];
                if (c == ' ' || c == '\t' || c == ',') { i++; continue; }
                if (c == '/') { slash = true; break; }
                size_t j = i;
                while (j < rec.size() && rec[j] != ' ' && rec[j] != '\t' && rec[j] != ',' && rec[j] != '/') j++;
                out.push_back(rec.substr(i, j - i));
                i = j;
            }
            if (slash) break;
        }
        return out;
    }
    std::vector<double> read_reals(size_t n) {
        std::vector<std::string> t = read_tokens(n);
        if (t.size() < n) throw DeckError("too few values in '" + path_ + "'");
        std::vector<double> v;
        for (auto& s : t) v.push_back(to_real(s));
        return v;
    }
    std::vector<long> read_ints(size_t n) {
        std::vector<std::string> t = read_tokens(n);
        if (t.size() < n) throw DeckError("too few values in '" + path_ + "'");
        std::vector<long> v;
        for (auto& s : t) v.push_back(to_int(s));
        return v;
    }
    double to_real(std::string s) const {
        for (auto& c : s)
            if (c == 'd' || c == 'D') c = 'e';
        char* end = nullptr;
        double v = std::strtod(s.c_str(), &end);
        if (end == s.c_str() || *end != '\0') throw DeckError("bad real '" + s + "' in '" + path_ + "'");
        return v;
    }
    long to_int(const std::string& s) const {
        char* end = nullptr;
        long v = std::strtol(s.c_str(), &end, 10);
        if (end == s.c_str() || *end != '\0') throw DeckError("bad integer '" + s + "' in '" + path_ + "'");
        return v;
    }
    const std::string& path() const { return path_; }

private:
    std::string path_;
    std::vector<std::string> lines_;
    size_t pos_ = 0;
};

inline std::string trim(const std::string& s) {
    size_t a = s.find_first_not_of(" \t");
    if (a == std::string::npos) return "";
    size_t b = s.find_last_not_of(" \t");
    return s.substr(a, b - a + 1);
}

}  // namespace orc
