// Fortran list-directed input reader for BELLHOP input files.
//
// Semantics follow the reference's LDIFile (src/util/ldio.hpp:42-410):
//  * record(): starts a new record; the rest of the current line is skipped
//    unless the reader is already at the start of a line;
//  * values are separated by blanks or one comma, may continue onto following
//    lines, and ',,' gives a null value (the destination keeps its value);
//  * '/' ends the record: every later read in it is null;
//  * 'text' or "text" are strings, (re,im) a complex number, n*v repeats v;
//  * doubles parse with strtod, floats with strtof (as the reference does).
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>

namespace bhcb {

class LdiReader {
public:
    explicit LdiReader(const std::string &path);
    bool good() const { return ok_; }
    void record();
    // Each returns false (leaving v unchanged) for a null value.
    bool read(double &v);
    bool read(float &v);
    bool read(int32_t &v);
    bool read(std::string &v);
    bool read_chars(char *v, size_t n);   // blank-padded to n
    const std::string &path() const { return path_; }

private:
    bool next_item(std::string &out);
    [[noreturn]] void fail(const std::string &msg) const;
    std::string buf_, path_, last_;
    size_t pos_ = 0;
    int line_ = 1;
    int repeat_ = 0;
    bool ok_ = false, after_slash_ = false, at_line_start_ = true;
};

} // namespace bhcb
