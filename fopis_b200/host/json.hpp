// json.hpp — the small JSON reader the host side needs for input.json.
//
// The reference parses input.json with picojson, whose objects are std::map
// (keys in sorted order); Value keeps the same ordering so species and objects
// come out in the order the reference iterates them. Numbers are doubles.
#pragma once

#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace fopis {
namespace host {

class Value {
public:
    enum class Kind { Null, Bool, Number, String, Array, Object };

    Value() = default;
    static Value parse(const std::string& text);
    static Value parse_file(const std::string& path);

    Kind kind() const { return kind_; }
    bool is_object() const { return kind_ == Kind::Object; }
    bool has(const std::string& key) const { return kind_ == Kind::Object && object_.count(key) != 0; }
    const Value& operator[](const std::string& key) const;
    const Value& operator[](size_t i) const;
    size_t size() const { return kind_ == Kind::Array ? array_.size() : object_.size(); }
    const std::map<std::string, Value>& items() const;

    double number() const;
    int integer() const;
    bool boolean() const;
    const std::string& str() const;

    double number_or(const std::string& key, double fallback) const { return has(key) ? (*this)[key].number() : fallback; }
    int integer_or(const std::string& key, int fallback) const { return has(key) ? (*this)[key].integer() : fallback; }
    bool boolean_or(const std::string& key, bool fallback) const { return has(key) ? (*this)[key].boolean() : fallback; }
    std::string str_or(const std::string& key, const std::string& fallback) const {
        return has(key) ? (*this)[key].str() : fallback;
    }

private:
    friend class Parser;
    Kind kind_ = Kind::Null;
    bool bool_ = false;
    double number_ = 0.0;
    std::string string_;
    std::vector<Value> array_;
    std::map<std::string, Value> object_;
};

}  // namespace host
}  // namespace fopis
