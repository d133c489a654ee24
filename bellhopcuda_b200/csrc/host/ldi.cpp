#include "ldi.h"

#include <cctype>
#include <cstdlib>
#include <fstream>
#include <sstream>

namespace bhcb {

LdiReader::LdiReader(const std::string &path) : path_(path)
{
    std::ifstream f(path, std::ios::binary);
    if(!f.good()) return;
    std::stringstream ss;
    ss << f.rdbuf();
    buf_ = ss.str();
    ok_ = true;
}

void LdiReader::fail(const std::string &msg) const
{
    throw std::runtime_error(path_ + ":" + std::to_string(line_) + ": " + msg);
}

void LdiReader::record()
{
    after_slash_ = false;
    repeat_ = 0;
    if(!at_line_start_) {
        while(pos_ < buf_.size() && buf_[pos_] != '\n') ++pos_;
        if(pos_ < buf_.size()) ++pos_;
        ++line_;
        at_line_start_ = true;
    }
}

// Returns false for a null item (after '/', an empty comma slot, or EOF).
bool LdiReader::next_item(std::string &out)
{
    if(repeat_ > 0) {
        --repeat_;
        out = last_;
        return true;
    }
    if(after_slash_) return false;
    while(pos_ < buf_.size() && isspace((unsigned char)buf_[pos_])) {
        if(buf_[pos_] == '\n') { ++line_; at_line_start_ = true; }
        else at_line_start_ = false;
        ++pos_;
    }
    if(pos_ >= buf_.size()) return false;
    if(buf_[pos_] == ',') {
        ++pos_;
        at_line_start_ = false;
        return false;
    }
    std::string item;
    int quote = 0; // 1 ", 2 ', 3 (
    bool closed_quote = false;
    while(pos_ < buf_.size()) {
        char c = buf_[pos_++];
        at_line_start_ = false;
        if(quote == 1 || quote == 2) {
            if((quote == 1 && c == '"') || (quote == 2 && c == '\'')) {
                quote = 0;
                closed_quote = true;
                break;
            }
            if(c == '\n') { ++line_; at_line_start_ = true; break; }
            item += c;
            continue;
        }
        if(c == '"') { quote = 1; continue; }
        if(c == '\'') { quote = 2; continue; }
        if(c == '(') { quote = 3; item += c; continue; }
        if(c == ')' && quote == 3) { item += c; quote = 0; closed_quote = true; break; }
        if(quote == 3) { item += c; continue; }
        if(isspace((unsigned char)c)) {
            if(c == '\n') { ++line_; at_line_start_ = true; }
            break;
        }
        if(c == ',') break;
        if(c == '*') {
            char *end = nullptr;
            long n = strtol(item.c_str(), &end, 10);
            if(item.empty() || *end || n <= 0) fail("invalid repetition count '" + item + "'");
            repeat_ = (int)n;
            item.clear();
            continue;
        }
        if(c == '/') {
            after_slash_ = true;
            break;
        }
        item += c;
    }
    if(quote != 0) fail("unterminated quote or parenthesis");
    (void)closed_quote;
    // consume trailing blanks and at most one comma / a slash
    if(!after_slash_ && !at_line_start_) {
        bool comma = false;
        while(pos_ < buf_.size()) {
            char c = buf_[pos_];
            if(c == '\n') { ++pos_; ++line_; at_line_start_ = true; break; }
            if(isspace((unsigned char)c)) { ++pos_; continue; }
            if(c == ',' && !comma) { ++pos_; comma = true; continue; }
            if(c == '/') { ++pos_; after_slash_ = true; }
            break;
        }
    }
    if(repeat_ > 0) {
        --repeat_;
        last_ = item;
    }
    out = item;
    return true;
}

bool LdiReader::read(double &v)
{
    std::string s;
    if(!next_item(s)) return false;
    char *end = nullptr;
    double d = strtod(s.c_str(), &end);
    if(s.empty() || *end) fail("'" + s + "' is not a real number");
    v = d;
    return true;
}

bool LdiReader::read(float &v)
{
    std::string s;
    if(!next_item(s)) return false;
    char *end = nullptr;
    float d = strtof(s.c_str(), &end);
    if(s.empty() || *end) fail("'" + s + "' is not a real number");
    v = d;
    return true;
}

bool LdiReader::read(int32_t &v)
{
    std::string s;
    if(!next_item(s)) return false;
    char *end = nullptr;
    long d = strtol(s.c_str(), &end, 10);
    if(s.empty() || *end) fail("'" + s + "' is not an integer");
    v = (int32_t)d;
    return true;
}

bool LdiReader::read(std::string &v)
{
    std::string s;
    if(!next_item(s)) return false;
    v = s;
    return true;
}

bool LdiReader::read_chars(char *v, size_t n)
{
    std::string s;
    if(!next_item(s)) return false;
    if(s.size() > n) fail("string '" + s + "' longer than " + std::to_string(n));
    for(size_t i = 0; i < n; ++i) v[i] = i < s.size() ? s[i] : ' ';
    return true;
}

} // namespace bhcb
