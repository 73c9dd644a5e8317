// json.cpp — recursive-descent JSON reader (RFC 8259 values; \uXXXX escapes
// below U+0080 decoded, others kept as '?', which input.json never needs).
#include "json.hpp"

#include <cctype>
#include <cstdlib>
#include <fstream>
#include <sstream>

namespace fopis {
namespace host {

namespace {
const Value& null_value() {
    static const Value v;
    return v;
}
}  // namespace

class Parser {
public:
    explicit Parser(const std::string& s) : s_(s) {}

    Value document() {
        Value v = value();
        ws();
        if (p_ != s_.size()) fail("trailing characters");
        return v;
    }

private:
    const std::string& s_;
    size_t p_ = 0;

    [[noreturn]] void fail(const std::string& what) const {
        throw std::runtime_error("input.json: " + what + " at offset " + std::to_string(p_));
    }
    void ws() {
        while (p_ < s_.size() && std::isspace((unsigned char)s_[p_])) ++p_;
    }
    bool take(char c) {
        ws();
        if (p_ < s_.size() && s_[p_] == c) { ++p_; return true; }
        return false;
    }
    void expect(char c) {
        if (!take(c)) fail(std::string("expected '") + c + "'");
    }
    bool literal(const char* word) {
        const std::string w(word);
        if (s_.compare(p_, w.size(), w) == 0) { p_ += w.size(); return true; }
        return false;
    }

    Value value() {
        ws();
        if (p_ >= s_.size()) fail("unexpected end");
        Value v;
        const char c = s_[p_];
        if (c == '{') {
            ++p_;
            v.kind_ = Value::Kind::Object;
            if (take('}')) return v;
            do {
                ws();
                const std::string key = string();
                expect(':');
                v.object_[key] = value();
            } while (take(','));
            expect('}');
        } else if (c == '[') {
            ++p_;
            v.kind_ = Value::Kind::Array;
            if (take(']')) return v;
            do { v.array_.push_back(value()); } while (take(','));
            expect(']');
        } else if (c == '"') {
            v.kind_ = Value::Kind::String;
            v.string_ = string();
        } else if (literal("true")) {
            v.kind_ = Value::Kind::Bool;
            v.bool_ = true;
        } else if (literal("false")) {
            v.kind_ = Value::Kind::Bool;
            v.bool_ = false;
        } else if (literal("null")) {
            v.kind_ = Value::Kind::Null;
        } else {
            v.kind_ = Value::Kind::Number;
            const char* begin = s_.c_str() + p_;
            char* end = nullptr;
            v.number_ = std::strtod(begin, &end);
            if (end == begin) fail("bad value");
            p_ += (size_t)(end - begin);
        }
        return v;
    }

    std::string string() {
        if (p_ >= s_.size() || s_[p_] != '"') fail("expected a string");
        ++p_;
        std::string out;
        while (p_ < s_.size() && s_[p_] != '"') {
            char c = s_[p_++];
            if (c == '\\') {
                if (p_ >= s_.size()) fail("bad escape");
                const char e = s_[p_++];
                switch (e) {
                    case 'n': out += '\n'; break;
                    case 't': out += '\t'; break;
                    case 'r': out += '\r'; break;
                    case 'b': out += '\b'; break;
                    case 'f': out += '\f'; break;
                    case 'u': {
                        if (p_ + 4 > s_.size()) fail("bad \\u escape");
                        const unsigned code = (unsigned)std::strtoul(s_.substr(p_, 4).c_str(), nullptr, 16);
                        p_ += 4;
                        out += code < 0x80 ? (char)code : '?';
                        break;
                    }
                    default: out += e;
                }
            } else {
                out += c;
            }
        }
        if (p_ >= s_.size()) fail("unterminated string");
        ++p_;
        return out;
    }
};

Value Value::parse(const std::string& text) { return Parser(text).document(); }

Value Value::parse_file(const std::string& path) {
    std::ifstream in(path);
    if (!in) throw std::runtime_error("cannot open " + path);
    std::stringstream ss;
    ss << in.rdbuf();
    return parse(ss.str());
}

const Value& Value::operator[](const std::string& key) const {
    if (kind_ != Kind::Object) throw std::runtime_error("input.json: '" + key + "' looked up in a non-object");
    const auto it = object_.find(key);
    if (it == object_.end()) throw std::runtime_error("input.json: missing key '" + key + "'");
    return it->second;
}
const Value& Value::operator[](size_t i) const {
    if (kind_ != Kind::Array || i >= array_.size()) return null_value();
    return array_[i];
}
const std::map<std::string, Value>& Value::items() const {
    if (kind_ != Kind::Object) throw std::runtime_error("input.json: expected an object");
    return object_;
}
double Value::number() const {
    if (kind_ == Kind::Bool) return bool_ ? 1.0 : 0.0;
    if (kind_ != Kind::Number) throw std::runtime_error("input.json: expected a number");
    return number_;
}
int Value::integer() const { return (int)number(); }
bool Value::boolean() const {
    if (kind_ == Kind::Number) return number_ != 0.0;
    if (kind_ != Kind::Bool) throw std::runtime_error("input.json: expected true/false");
    return bool_;
}
const std::string& Value::str() const {
    if (kind_ != Kind::String) throw std::runtime_error("input.json: expected a string");
    return string_;
}

}  // namespace host
}  // namespace fopis
