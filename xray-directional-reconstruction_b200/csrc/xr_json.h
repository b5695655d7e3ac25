/*
 * A small JSON reader for the reference's settings.json schema
 * (utility/settings.json: objects, arrays, numbers, strings, booleans).
 * The reference parses the file with the vendored nlohmann/json
 * (params.cu:44); this is a separate, minimal recursive-descent parser.
 */
#ifndef XR_JSON_H
#define XR_JSON_H

#include <cstdlib>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

namespace xr {

struct JVal {
    enum Kind { Null, Bool, Num, Str, Arr, Obj } kind = Null;
    bool b = false;
    double n = 0.0;
    std::string s;
    std::vector<JVal> a;
    std::vector<std::pair<std::string, JVal>> o;

    const JVal *get(const std::string &key) const {
        if (kind != Obj) return nullptr;
        for (const auto &kv : o)
            if (kv.first == key) return &kv.second;
        return nullptr;
    }
};

class JParser {
  public:
    JParser(const char *p, const char *end) : p_(p), end_(end) {}

    bool parse(JVal &out, std::string &err) {
        if (!value(out, 0)) {
            err = err_.empty() ? "malformed JSON" : err_;
            return false;
        }
        ws();
        if (p_ != end_) {
            err = "trailing characters after JSON value";
            return false;
        }
        return true;
    }

  private:
    const char *p_, *end_;
    std::string err_;

    void ws() {
        while (p_ < end_ && (*p_ == ' ' || *p_ == '\n' || *p_ == '\r' || *p_ == '\t')) ++p_;
    }
    bool fail(const char *m) {
        if (err_.empty()) err_ = m;
        return false;
    }
    bool lit(const char *w) {
        const char *q = p_;
        for (; *w; ++w, ++q)
            if (q >= end_ || *q != *w) return false;
        p_ = q;
        return true;
    }
    bool str(std::string &out) {
        if (p_ >= end_ || *p_ != '"') return fail("expected string");
        ++p_;
        while (p_ < end_ && *p_ != '"') {
            char c = *p_++;
            if (c == '\\') {
                if (p_ >= end_) return fail("bad escape");
                const char e = *p_++;
                switch (e) {
                    case 'n': out += '\n'; break;
                    case 't': out += '\t'; break;
                    case 'r': out += '\r'; break;
                    case 'b': out += '\b'; break;
                    case 'f': out += '\f'; break;
                    case 'u': {
                        if (end_ - p_ < 4) return fail("bad \\u escape");
                        const unsigned cp = (unsigned)std::strtoul(std::string(p_, p_ + 4).c_str(), nullptr, 16);
                        p_ += 4;
                        if (cp < 0x80) out += (char)cp;
                        else if (cp < 0x800) { out += (char)(0xC0 | (cp >> 6)); out += (char)(0x80 | (cp & 0x3F)); }
                        else { out += (char)(0xE0 | (cp >> 12)); out += (char)(0x80 | ((cp >> 6) & 0x3F));
                               out += (char)(0x80 | (cp & 0x3F)); }
                        break;
                    }
                    default: out += e; break;
                }
            } else {
                out += c;
            }
        }
        if (p_ >= end_) return fail("unterminated string");
        ++p_;
        return true;
    }
    bool value(JVal &v, int depth) {
        if (depth > 64) return fail("JSON nested too deeply");
        ws();
        if (p_ >= end_) return fail("unexpected end of JSON");
        const char c = *p_;
        if (c == '{') {
            ++p_;
            v.kind = JVal::Obj;
            ws();
            if (p_ < end_ && *p_ == '}') { ++p_; return true; }
            for (;;) {
                ws();
                std::string k;
                if (!str(k)) return false;
                ws();
                if (p_ >= end_ || *p_ != ':') return fail("expected ':'");
                ++p_;
                JVal child;
                if (!value(child, depth + 1)) return false;
                v.o.emplace_back(std::move(k), std::move(child));
                ws();
                if (p_ < end_ && *p_ == ',') { ++p_; continue; }
                if (p_ < end_ && *p_ == '}') { ++p_; return true; }
                return fail("expected ',' or '}'");
            }
        }
        if (c == '[') {
            ++p_;
            v.kind = JVal::Arr;
            ws();
            if (p_ < end_ && *p_ == ']') { ++p_; return true; }
            for (;;) {
                JVal child;
                if (!value(child, depth + 1)) return false;
                v.a.push_back(std::move(child));
                ws();
                if (p_ < end_ && *p_ == ',') { ++p_; continue; }
                if (p_ < end_ && *p_ == ']') { ++p_; return true; }
                return fail("expected ',' or ']'");
            }
        }
        if (c == '"') { v.kind = JVal::Str; return str(v.s); }
        if (lit("true")) { v.kind = JVal::Bool; v.b = true; return true; }
        if (lit("false")) { v.kind = JVal::Bool; v.b = false; return true; }
        if (lit("null")) { v.kind = JVal::Null; return true; }
        if (c == '-' || (c >= '0' && c <= '9')) {
            std::string num;
            while (p_ < end_ && *p_ != '\0' && std::strchr("+-0123456789.eE", *p_) != nullptr) num += *p_++;
            char *e = nullptr;
            v.kind = JVal::Num;
            v.n = std::strtod(num.c_str(), &e);
            if (e == num.c_str() || *e != '\0') return fail("bad number");
            return true;
        }
        return fail("unexpected character in JSON");
    }
};

}  // namespace xr

#endif
