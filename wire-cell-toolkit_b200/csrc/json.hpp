// Minimal JSON reader for component configuration (the subset produced by
// Jsonnet -> JSON in Wire-Cell configurations: objects, arrays, strings,
// numbers, booleans, null).  Numbers follow the JSON grammar and convert
// independently of the process locale (a host framework may set LC_NUMERIC);
// nesting deeper than kMaxDepth is refused instead of exhausting the stack.
#pragma once

#include <cctype>
#include <charconv>
#include <cstdlib>
#include <system_error>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace wctb200 {
namespace json {

struct Value {
    enum Kind { Null, Bool, Number, String, Array, Object } kind{Null};
    bool b{false};
    double num{0};
    std::string str;
    std::vector<Value> arr;
    std::map<std::string, Value> obj;

    bool is_null() const { return kind == Null; }
    bool has(const std::string& k) const { return kind == Object && obj.count(k); }
    const Value& operator[](const std::string& k) const
    {
        static const Value null;
        if (kind != Object) return null;
        auto it = obj.find(k);
        return it == obj.end() ? null : it->second;
    }
    double as_number(double dflt) const
    {
        if (kind == Number) return num;
        if (kind == Bool) return b ? 1.0 : 0.0;
        return dflt;
    }
    bool as_bool(bool dflt) const
    {
        if (kind == Bool) return b;
        if (kind == Number) return num != 0.0;
        return dflt;
    }
    std::string as_string(const std::string& dflt) const { return kind == String ? str : dflt; }
};

class Parser {
   public:
    explicit Parser(const std::string& s) : s_(s) {}
    Value parse()
    {
        Value v = value();
        ws();
        if (i_ != s_.size()) fail("trailing characters");
        return v;
    }

    static constexpr int kMaxDepth = 256;

   private:
    const std::string& s_;
    size_t i_{0};
    int depth_{0};
    [[noreturn]] void fail(const char* what)
    {
        throw std::runtime_error(std::string("json: ") + what + " at offset " + std::to_string(i_));
    }
    void ws()
    {
        while (i_ < s_.size() && std::isspace((unsigned char)s_[i_])) ++i_;
    }
    bool eat(char c)
    {
        ws();
        if (i_ < s_.size() && s_[i_] == c) { ++i_; return true; }
        return false;
    }
    Value value()
    {
        ws();
        if (i_ >= s_.size()) fail("unexpected end");
        const char c = s_[i_];
        if (c == '{') return object();
        if (c == '[') return array();
        if (c == '"') { Value v; v.kind = Value::String; v.str = string(); return v; }
        if (s_.compare(i_, 4, "true") == 0) { i_ += 4; Value v; v.kind = Value::Bool; v.b = true; return v; }
        if (s_.compare(i_, 5, "false") == 0) { i_ += 5; Value v; v.kind = Value::Bool; v.b = false; return v; }
        if (s_.compare(i_, 4, "null") == 0) { i_ += 4; return Value{}; }
        return number();
    }
    Value number()
    {
        // -?(0|[1-9][0-9]*)(.[0-9]+)?([eE][+-]?[0-9]+)?
        const size_t n = s_.size();
        size_t j = i_;
        auto digits = [&]() {
            const size_t k = j;
            while (j < n && s_[j] >= '0' && s_[j] <= '9') ++j;
            return j > k;
        };
        if (j < n && s_[j] == '-') ++j;
        if (j < n && s_[j] == '0') ++j;
        else if (!digits()) fail("bad value");
        if (j < n && s_[j] == '.') {
            ++j;
            if (!digits()) fail("bad number");
        }
        if (j < n && (s_[j] == 'e' || s_[j] == 'E')) {
            ++j;
            if (j < n && (s_[j] == '+' || s_[j] == '-')) ++j;
            if (!digits()) fail("bad number");
        }
        double d = 0.0;
        const auto r = std::from_chars(s_.data() + i_, s_.data() + j, d);
        if (r.ec != std::errc() || r.ptr != s_.data() + j) fail("number out of range");
        i_ = j;
        Value v;
        v.kind = Value::Number;
        v.num = d;
        return v;
    }
    std::string string()
    {
        if (s_[i_] != '"') fail("expected string");
        ++i_;
        std::string out;
        while (i_ < s_.size() && s_[i_] != '"') {
            char c = s_[i_++];
            if (c == '\\') {
                if (i_ >= s_.size()) fail("bad escape");
                char e = s_[i_++];
                switch (e) {
                    case 'n': out += '\n'; break;
                    case 't': out += '\t'; break;
                    case 'r': out += '\r'; break;
                    case 'b': out += '\b'; break;
                    case 'f': out += '\f'; break;
                    case 'u': {
                        if (i_ + 4 > s_.size()) fail("bad unicode escape");
                        unsigned cp = std::strtoul(s_.substr(i_, 4).c_str(), nullptr, 16);
                        i_ += 4;
                        if (cp < 0x80) out += (char)cp;
                        else if (cp < 0x800) { out += (char)(0xC0 | (cp >> 6)); out += (char)(0x80 | (cp & 0x3F)); }
                        else {
                            out += (char)(0xE0 | (cp >> 12));
                            out += (char)(0x80 | ((cp >> 6) & 0x3F));
                            out += (char)(0x80 | (cp & 0x3F));
                        }
                        break;
                    }
                    default: out += e;
                }
            }
            else out += c;
        }
        if (i_ >= s_.size()) fail("unterminated string");
        ++i_;
        return out;
    }
    Value array()
    {
        if (++depth_ > kMaxDepth) fail("nesting too deep");
        Value v;
        v.kind = Value::Array;
        eat('[');
        if (!eat(']')) {
            do { v.arr.push_back(value()); } while (eat(','));
            if (!eat(']')) fail("expected ]");
        }
        --depth_;
        return v;
    }
    Value object()
    {
        if (++depth_ > kMaxDepth) fail("nesting too deep");
        Value v;
        v.kind = Value::Object;
        eat('{');
        if (!eat('}')) {
            do {
                ws();
                std::string k = string();
                if (!eat(':')) fail("expected :");
                v.obj[k] = value();
            } while (eat(','));
            if (!eat('}')) fail("expected }");
        }
        --depth_;
        return v;
    }
};

inline Value parse(const std::string& s) { return Parser(s).parse(); }

}  // namespace json
}  // namespace wctb200
