// json.cpp — parser and writers for fps::Json (see json.h).
#include "json.h"

#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>

namespace fps {

static const Json kNull;

double Json::asDouble() const
{
    switch (type_) {
        case Int: return (double)i_;
        case Real: return d_;
        case Bool: return b_ ? 1.0 : 0.0;
        case String: return std::strtod(s_.c_str(), nullptr);
        default: return 0.0;
    }
}

long long Json::asInt() const
{
    switch (type_) {
        case Int: return i_;
        case Real: return (long long)d_;
        case Bool: return b_ ? 1 : 0;
        case String: return std::strtoll(s_.c_str(), nullptr, 10);
        default: return 0;
    }
}

bool Json::asBool() const
{
    switch (type_) {
        case Bool: return b_;
        case Int: return i_ != 0;
        case Real: return d_ != 0.0;
        case String: return !s_.empty();
        default: return false;
    }
}

std::string Json::asString() const
{
    switch (type_) {
        case String: return s_;
        case Bool: return b_ ? "true" : "false";
        case Int: return std::to_string(i_);
        case Real: return json_number(d_);
        default: return "";
    }
}

size_t Json::size() const
{
    if (type_ == Array) return arr_.size();
    if (type_ == Object) return obj_.size();
    return 0;
}

bool Json::isMember(const std::string& key) const { return type_ == Object && obj_.count(key) > 0; }

Json& Json::operator[](const std::string& key)
{
    if (type_ == Null) type_ = Object;
    return obj_[key];
}

const Json& Json::operator[](const std::string& key) const
{
    if (type_ != Object) return kNull;
    auto it = obj_.find(key);
    return it == obj_.end() ? kNull : it->second;
}

Json& Json::operator[](size_t i)
{
    if (type_ == Null) type_ = Array;
    if (i >= arr_.size()) arr_.resize(i + 1);
    return arr_[i];
}

const Json& Json::operator[](size_t i) const
{
    if (type_ != Array || i >= arr_.size()) return kNull;
    return arr_[i];
}

Json& Json::append(const Json& v)
{
    if (type_ == Null) type_ = Array;
    arr_.push_back(v);
    return arr_.back();
}

Json Json::get(const std::string& key, const Json& dflt) const
{
    if (type_ != Object) return dflt;
    auto it = obj_.find(key);
    return it == obj_.end() ? dflt : it->second;
}

bool Json::operator==(const Json& o) const
{
    if (isNumber() && o.isNumber()) return asDouble() == o.asDouble();
    if (type_ != o.type_) return false;
    switch (type_) {
        case Null: return true;
        case Bool: return b_ == o.b_;
        case String: return s_ == o.s_;
        case Array: return arr_ == o.arr_;
        case Object: return obj_ == o.obj_;
        default: return false;
    }
}

// ------------------------------------------------------------------ parser
namespace {

struct Parser {
    const std::string& t;
    size_t p = 0;
    std::string err;
    explicit Parser(const std::string& s) : t(s) {}

    void skip()
    {
        for (;;) {
            while (p < t.size() && (t[p] == ' ' || t[p] == '\t' || t[p] == '\n' || t[p] == '\r')) ++p;
            if (p + 1 < t.size() && t[p] == '/' && t[p + 1] == '/') {
                while (p < t.size() && t[p] != '\n') ++p;
            } else if (p + 1 < t.size() && t[p] == '/' && t[p + 1] == '*') {
                const size_t e = t.find("*/", p + 2);
                p = (e == std::string::npos) ? t.size() : e + 2;
            } else {
                break;
            }
        }
    }
    bool fail(const std::string& m)
    {
        if (err.empty()) {
            size_t line = 1;
            for (size_t q = 0; q < p && q < t.size(); ++q) line += t[q] == '\n';
            err = m + " at line " + std::to_string(line);
        }
        return false;
    }
    bool lit(const char* w)
    {
        const size_t n = std::strlen(w);
        if (t.compare(p, n, w) == 0) { p += n; return true; }
        return false;
    }
    bool str(std::string& out)
    {
        if (p >= t.size() || t[p] != '"') return fail("expected a string");
        ++p;
        out.clear();
        while (p < t.size() && t[p] != '"') {
            char c = t[p++];
            if (c == '\\') {
                if (p >= t.size()) return fail("bad escape");
                char e = t[p++];
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
                        if (p + 4 > t.size()) return fail("bad \\u escape");
                        unsigned cp = (unsigned)std::stoul(t.substr(p, 4), nullptr, 16);
                        p += 4;
                        if (cp < 0x80) out += (char)cp;
                        else if (cp < 0x800) { out += (char)(0xC0 | (cp >> 6)); out += (char)(0x80 | (cp & 0x3F)); }
                        else { out += (char)(0xE0 | (cp >> 12)); out += (char)(0x80 | ((cp >> 6) & 0x3F)); out += (char)(0x80 | (cp & 0x3F)); }
                        break;
                    }
                    default: return fail("bad escape");
                }
            } else {
                out += c;
            }
        }
        if (p >= t.size()) return fail("unterminated string");
        ++p;
        return true;
    }
    bool value(Json& out, int depth)
    {
        if (depth > 512) return fail("nesting too deep");
        skip();
        if (p >= t.size()) return fail("unexpected end of input");
        const char c = t[p];
        if (c == '{') {
            ++p;
            out = Json::object();
            skip();
            if (p < t.size() && t[p] == '}') { ++p; return true; }
            for (;;) {
                skip();
                std::string key;
                if (!str(key)) return false;
                skip();
                if (p >= t.size() || t[p] != ':') return fail("expected ':'");
                ++p;
                Json v;
                if (!value(v, depth + 1)) return false;
                out[key] = v;
                skip();
                if (p < t.size() && t[p] == ',') { ++p; continue; }
                if (p < t.size() && t[p] == '}') { ++p; return true; }
                return fail("expected ',' or '}'");
            }
        }
        if (c == '[') {
            ++p;
            out = Json::array();
            skip();
            if (p < t.size() && t[p] == ']') { ++p; return true; }
            for (;;) {
                Json v;
                if (!value(v, depth + 1)) return false;
                out.append(v);
                skip();
                if (p < t.size() && t[p] == ',') { ++p; continue; }
                if (p < t.size() && t[p] == ']') { ++p; return true; }
                return fail("expected ',' or ']'");
            }
        }
        if (c == '"') {
            std::string s;
            if (!str(s)) return false;
            out = Json(s);
            return true;
        }
        if (lit("true")) { out = Json(true); return true; }
        if (lit("false")) { out = Json(false); return true; }
        if (lit("null")) { out = Json(); return true; }
        // number
        const size_t s0 = p;
        if (p < t.size() && (t[p] == '-' || t[p] == '+')) ++p;
        bool real = false;
        while (p < t.size() && (std::isdigit((unsigned char)t[p]) || t[p] == '.' || t[p] == 'e' || t[p] == 'E' ||
                                ((t[p] == '-' || t[p] == '+') && (t[p - 1] == 'e' || t[p - 1] == 'E')))) {
            if (t[p] == '.' || t[p] == 'e' || t[p] == 'E') real = true;
            ++p;
        }
        if (p == s0) return fail(std::string("unexpected character '") + c + "'");
        const std::string num = t.substr(s0, p - s0);
        char* end = nullptr;
        if (!real) {
            errno = 0;
            const long long v = std::strtoll(num.c_str(), &end, 10);
            if (errno == 0 && end && *end == '\0') { out = Json(v); return true; }
        }
        const double d = std::strtod(num.c_str(), &end);
        if (!end || *end != '\0') return fail("malformed number");
        out = Json(d);
        return true;
    }
};

}  // namespace

bool Json::parse(const std::string& text, Json& out, std::string& err)
{
    Parser ps(text);
    Json v;
    if (!ps.value(v, 0)) { err = ps.err; return false; }
    ps.skip();
    if (ps.p != text.size()) { err = "trailing characters after the document"; return false; }
    out = v;
    return true;
}

bool Json::parseFile(const std::string& path, Json& out, std::string& err)
{
    std::ifstream f(path);
    if (!f.good()) { err = path + " not found"; return false; }
    std::stringstream ss;
    ss << f.rdbuf();
    return parse(ss.str(), out, err);
}

// ------------------------------------------------------------------ writers
std::string json_number(double v)
{
    if (std::isnan(v)) return "null";
    if (std::isinf(v)) return v > 0 ? "1e+9999" : "-1e+9999";
    char buf[40];
    std::snprintf(buf, sizeof(buf), "%.17g", v);
    std::string s(buf);
    if (s.find('.') == std::string::npos && s.find('e') == std::string::npos) s += ".0";
    return s;
}

std::string json_quote(const std::string& s)
{
    std::string o = "\"";
    for (char c : s) {
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
                    char b[8];
                    std::snprintf(b, sizeof(b), "\\u%04x", (unsigned char)c);
                    o += b;
                } else {
                    o += c;
                }
        }
    }
    return o + "\"";
}

struct JsonWriter {
    std::string out;
    std::string indent;
    static constexpr size_t kRightMargin = 74;

    static std::string scalar(const Json& v)
    {
        switch (v.type_) {
            case Json::Null: return "null";
            case Json::Bool: return v.b_ ? "true" : "false";
            case Json::Int: return std::to_string(v.i_);
            case Json::Real: return json_number(v.d_);
            case Json::String: return json_quote(v.s_);
            case Json::Array: return v.arr_.empty() ? "[]" : "";
            case Json::Object: return v.obj_.empty() ? "{}" : "";
        }
        return "null";
    }
    void newline_indent() { out += '\n'; out += indent; }
    // a scalar array that fits the margin goes on one line: "[ a, b, c ]"
    bool one_line(const Json& v, std::vector<std::string>& parts)
    {
        if (v.arr_.size() * 3 >= kRightMargin) return false;
        size_t len = 4 + (v.arr_.size() - 1) * 2;
        for (const Json& c : v.arr_) {
            if ((c.type_ == Json::Array || c.type_ == Json::Object) && c.size() > 0) return false;
            parts.push_back(scalar(c));
            len += parts.back().size();
        }
        return len < kRightMargin;
    }
    void value(const Json& v)
    {
        if (v.type_ == Json::Object && !v.obj_.empty()) {
            newline_indent();
            out += '{';
            indent += '\t';
            size_t k = 0;
            for (const auto& kv : v.obj_) {
                newline_indent();
                out += json_quote(kv.first);
                out += " : ";
                value(kv.second);
                if (++k < v.obj_.size()) out += ',';
            }
            indent.pop_back();
            newline_indent();
            out += '}';
        } else if (v.type_ == Json::Array && !v.arr_.empty()) {
            std::vector<std::string> parts;
            if (one_line(v, parts)) {
                out += "[ ";
                for (size_t i = 0; i < parts.size(); ++i) {
                    if (i) out += ", ";
                    out += parts[i];
                }
                out += " ]";
                return;
            }
            newline_indent();
            out += '[';
            indent += '\t';
            for (size_t i = 0; i < v.arr_.size(); ++i) {
                const Json& c = v.arr_[i];
                std::vector<std::string> sub;
                if (c.type_ == Json::Object && !c.obj_.empty()) {
                    value(c);
                } else if (c.type_ == Json::Array && !c.arr_.empty()) {
                    if (one_line(c, sub)) newline_indent();
                    value(c);
                } else {
                    newline_indent();
                    out += scalar(c);
                }
                if (i + 1 < v.arr_.size()) out += ',';
            }
            indent.pop_back();
            newline_indent();
            out += ']';
        } else {
            out += scalar(v);
        }
    }
};

std::string Json::styled() const
{
    JsonWriter w;
    w.value(*this);
    std::string s = w.out;
    if (!s.empty() && s[0] == '\n') s.erase(0, 1);
    return s;
}

std::string Json::compact() const
{
    switch (type_) {
        case Array: {
            std::string s = "[";
            for (size_t i = 0; i < arr_.size(); ++i) s += (i ? "," : "") + arr_[i].compact();
            return s + "]";
        }
        case Object: {
            std::string s = "{";
            size_t k = 0;
            for (const auto& kv : obj_) s += (k++ ? "," : "") + json_quote(kv.first) + ":" + kv.second.compact();
            return s + "}";
        }
        default: return JsonWriter::scalar(*this);
    }
}

}  // namespace fps
