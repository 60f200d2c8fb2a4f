// json.h — the JSON value used by the host layer (input system files and result
// documents).  Semantics follow what FermiPhaseSpace relies on from jsoncpp
// (include/json/json.h): objects keep their keys sorted, integers and reals stay
// distinct, get(key, default) returns the default for absent keys, comments are
// accepted on input, and the styled writer indents with tabs, writes short scalar
// arrays on one line and reals with 17 significant digits.
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace fps {

class Json {
public:
    enum Type { Null, Bool, Int, Real, String, Array, Object };

    Json() = default;
    Json(std::nullptr_t) {}
    Json(bool b) : type_(Bool), b_(b) {}
    Json(int v) : type_(Int), i_(v) {}
    Json(unsigned v) : type_(Int), i_(v) {}
    Json(long v) : type_(Int), i_(v) {}
    Json(long long v) : type_(Int), i_(v) {}
    Json(unsigned long v) : type_(Int), i_((long long)v) {}
    Json(double v) : type_(Real), d_(v) {}
    Json(const char* s) : type_(String), s_(s) {}
    Json(const std::string& s) : type_(String), s_(s) {}
    static Json array() { Json j; j.type_ = Array; return j; }
    static Json object() { Json j; j.type_ = Object; return j; }

    Type type() const { return type_; }
    bool isNull() const { return type_ == Null; }
    bool isArray() const { return type_ == Array; }
    bool isObject() const { return type_ == Object; }
    bool isNumber() const { return type_ == Int || type_ == Real; }
    bool isString() const { return type_ == String; }
    bool isBool() const { return type_ == Bool; }

    double asDouble() const;
    long long asInt() const;
    unsigned asUInt() const { return (unsigned)asInt(); }
    bool asBool() const;
    std::string asString() const;

    size_t size() const;
    bool isMember(const std::string& key) const;
    // object access; a null value becomes an object on first write
    Json& operator[](const std::string& key);
    const Json& operator[](const std::string& key) const;
    // array access
    Json& operator[](size_t i);
    const Json& operator[](size_t i) const;
    Json& append(const Json& v);
    Json get(const std::string& key, const Json& dflt) const;
    const std::map<std::string, Json>& members() const { return obj_; }
    const std::vector<Json>& items() const { return arr_; }

    bool operator==(const Json& o) const;
    bool operator!=(const Json& o) const { return !(*this == o); }

    // parsing: returns false and sets err on malformed input
    static bool parse(const std::string& text, Json& out, std::string& err);
    static bool parseFile(const std::string& path, Json& out, std::string& err);
    // tab-indented styled document (jsoncpp StreamWriterBuilder, indentation "\t")
    std::string styled() const;
    // compact single-line form
    std::string compact() const;

private:
    Type type_ = Null;
    bool b_ = false;
    long long i_ = 0;
    double d_ = 0.0;
    std::string s_;
    std::vector<Json> arr_;
    std::map<std::string, Json> obj_;

    friend struct JsonWriter;
};

std::string json_number(double v);   // "%.17g", ".0" appended to integral-looking values
std::string json_quote(const std::string& s);

}  // namespace fps
