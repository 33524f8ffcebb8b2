// Strict recursive-descent JSON parser (RFC 8259) and string escaper (API: WVM/include/wf/json.hpp).
#include <cstdio>
#include <cstdlib>
#include <string>
#include "wf/json.hpp"

namespace wf {
namespace {

class Parser {
public:
    explicit Parser(const std::string& t) : t_(t) {}

    Json document() {
        ws();
        Json v = value(0);
        ws();
        if (i_ != t_.size()) fail("trailing characters after the document");
        return v;
    }

private:
    const std::string& t_;
    size_t i_ = 0;

    [[noreturn]] void fail(const std::string& what) const {
        throw std::runtime_error("json_parse: " + what + " at offset " + std::to_string(i_));
    }
    void ws() {
        while (i_ < t_.size() && (t_[i_] == ' ' || t_[i_] == '\t' || t_[i_] == '\n' || t_[i_] == '\r')) ++i_;
    }
    bool eat(char c) {
        if (i_ < t_.size() && t_[i_] == c) {
            ++i_;
            return true;
        }
        return false;
    }
    void expect_word(const char* w) {
        for (const char* p = w; *p; ++p)
            if (!eat(*p)) fail(std::string("invalid literal (expected ") + w + ")");
    }

    Json value(int depth) {
        if (depth > 512) fail("nesting too deep");
        if (i_ >= t_.size()) fail("unexpected end of input");
        Json v;
        const char c = t_[i_];
        if (c == '{') {
            ++i_;
            v.type = Json::Object;
            ws();
            if (eat('}')) return v;
            for (;;) {
                ws();
                if (i_ >= t_.size() || t_[i_] != '"') fail("expected a string key");
                std::string k = string_body();
                ws();
                if (!eat(':')) fail("expected ':'");
                ws();
                v.obj[k] = value(depth + 1);
                ws();
                if (eat(',')) continue;
                if (eat('}')) return v;
                fail("expected ',' or '}'");
            }
        }
        if (c == '[') {
            ++i_;
            v.type = Json::Array;
            ws();
            if (eat(']')) return v;
            for (;;) {
                ws();
                v.arr.push_back(value(depth + 1));
                ws();
                if (eat(',')) continue;
                if (eat(']')) return v;
                fail("expected ',' or ']'");
            }
        }
        if (c == '"') {
            v.type = Json::String;
            v.str = string_body();
            return v;
        }
        if (c == 't') {
            expect_word("true");
            v.type = Json::Bool;
            v.b = true;
            return v;
        }
        if (c == 'f') {
            expect_word("false");
            v.type = Json::Bool;
            return v;
        }
        if (c == 'n') {
            expect_word("null");
            return v;
        }
        if (c == '-' || (c >= '0' && c <= '9')) {
            v.type = Json::Number;
            v.num = number();
            return v;
        }
        fail(std::string("unexpected character '") + c + "'");
    }

    double number() {
        const size_t start = i_;
        eat('-');
        if (eat('0')) {
        } else if (i_ < t_.size() && t_[i_] >= '1' && t_[i_] <= '9') {
            while (i_ < t_.size() && t_[i_] >= '0' && t_[i_] <= '9') ++i_;
        } else {
            fail("malformed number");
        }
        if (eat('.')) {
            if (!(i_ < t_.size() && t_[i_] >= '0' && t_[i_] <= '9')) fail("malformed fraction");
            while (i_ < t_.size() && t_[i_] >= '0' && t_[i_] <= '9') ++i_;
        }
        if (i_ < t_.size() && (t_[i_] == 'e' || t_[i_] == 'E')) {
            ++i_;
            if (!eat('+')) eat('-');
            if (!(i_ < t_.size() && t_[i_] >= '0' && t_[i_] <= '9')) fail("malformed exponent");
            while (i_ < t_.size() && t_[i_] >= '0' && t_[i_] <= '9') ++i_;
        }
        return std::strtod(t_.substr(start, i_ - start).c_str(), nullptr);
    }

    unsigned hex4() {
        unsigned v = 0;
        for (int k = 0; k < 4; ++k) {
            if (i_ >= t_.size()) fail("truncated \\u escape");
            const char h = t_[i_++];
            v <<= 4;
            if (h >= '0' && h <= '9') v |= (unsigned)(h - '0');
            else if (h >= 'a' && h <= 'f') v |= (unsigned)(h - 'a' + 10);
            else if (h >= 'A' && h <= 'F') v |= (unsigned)(h - 'A' + 10);
            else fail("bad hex digit in \\u escape");
        }
        return v;
    }

    static void utf8(std::string& out, unsigned cp) {
        if (cp < 0x80) {
            out += (char)cp;
        } else if (cp < 0x800) {
            out += (char)(0xC0 | (cp >> 6));
            out += (char)(0x80 | (cp & 0x3F));
        } else if (cp < 0x10000) {
            out += (char)(0xE0 | (cp >> 12));
            out += (char)(0x80 | ((cp >> 6) & 0x3F));
            out += (char)(0x80 | (cp & 0x3F));
        } else {
            out += (char)(0xF0 | (cp >> 18));
            out += (char)(0x80 | ((cp >> 12) & 0x3F));
            out += (char)(0x80 | ((cp >> 6) & 0x3F));
            out += (char)(0x80 | (cp & 0x3F));
        }
    }

    std::string string_body() {
        ++i_;  // opening quote
        std::string out;
        for (;;) {
            if (i_ >= t_.size()) fail("unterminated string");
            const char c = t_[i_++];
            if (c == '"') return out;
            if ((unsigned char)c < 0x20) fail("control character in string");
            if (c != '\\') {
                out += c;
                continue;
            }
            if (i_ >= t_.size()) fail("unterminated escape");
            const char e = t_[i_++];
            switch (e) {
                case '"': out += '"'; break;
                case '\\': out += '\\'; break;
                case '/': out += '/'; break;
                case 'b': out += '\b'; break;
                case 'f': out += '\f'; break;
                case 'n': out += '\n'; break;
                case 'r': out += '\r'; break;
                case 't': out += '\t'; break;
                case 'u': {
                    unsigned cp = hex4();
                    if (cp >= 0xD800 && cp <= 0xDBFF && i_ + 1 < t_.size() && t_[i_] == '\\' && t_[i_ + 1] == 'u') {
                        const size_t save = i_;
                        i_ += 2;
                        const unsigned lo = hex4();
                        if (lo >= 0xDC00 && lo <= 0xDFFF) cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
                        else i_ = save;
                    }
                    utf8(out, cp);
                    break;
                }
                default: fail(std::string("bad escape \\") + e);
            }
        }
    }
};

}  // namespace

Json json_parse(const std::string& text) { return Parser(text).document(); }

std::string json_escape(const std::string& s) {
    std::string o;
    o.reserve(s.size() + 8);
    for (const char c : s) {
        switch (c) {
            case '"': o += "\\\""; break;
            case '\\': o += "\\\\"; break;
            case '\n': o += "\\n"; break;
            case '\r': o += "\\r"; break;
            case '\t': o += "\\t"; break;
            case '\b': o += "\\b"; break;
            case '\f': o += "\\f"; break;
            default:
                if ((unsigned char)c < 0x20) {
                    char buf[8];
                    std::snprintf(buf, sizeof buf, "\\u%04x", (unsigned)(unsigned char)c);
                    o += buf;
                } else {
                    o += c;
                }
        }
    }
    return o;
}

}  // namespace wf
