// Minimal JSON reader for the material / integrator / camera descriptions the C API accepts
// (objects, arrays, numbers, strings, booleans, null).
#pragma once

#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace spb::json {

struct Value {
    enum class Kind { Null, Bool, Number, String, Array, Object };

    Kind                                 kind = Kind::Null;
    bool                                 boolean = false;
    double                               number  = 0.0;
    std::string                          string;
    std::vector<Value>                   array;
    std::vector<std::pair<std::string, Value>> object;  // keeps member order

    Value const* find(std::string const& key) const {
        for (auto const& kv : object) {
            if (kv.first == key) {
                return &kv.second;
            }
        }
        return nullptr;
    }

    bool is_number() const {
        return kind == Kind::Number;
    }
    bool is_object() const {
        return kind == Kind::Object;
    }
    bool is_array() const {
        return kind == Kind::Array;
    }
    bool is_string() const {
        return kind == Kind::String;
    }
};

class Parser {
  public:
    explicit Parser(char const* text) : p_(text) {}

    bool parse(Value& out) {
        skip();
        if (!value(out)) {
            return false;
        }
        skip();
        return *p_ == '\0';
    }

  private:
    void skip() {
        while (*p_ && std::isspace(static_cast<unsigned char>(*p_))) {
            ++p_;
        }
    }

    bool literal(char const* word) {
        size_t i = 0;
        for (; word[i]; ++i) {
            if (p_[i] != word[i]) {
                return false;
            }
        }
        p_ += i;
        return true;
    }

    bool string_body(std::string& s) {
        ++p_;  // opening quote
        while (*p_ && *p_ != '"') {
            if (*p_ == '\\') {
                ++p_;
                switch (*p_) {
                    case 'n': s += '\n'; break;
                    case 't': s += '\t'; break;
                    case 'r': s += '\r'; break;
                    case 'b': s += '\b'; break;
                    case 'f': s += '\f'; break;
                    case 'u':
                        // keep \uXXXX escapes verbatim; the descriptions use plain ASCII keys
                        s += "\\u";
                        break;
                    case '\0': return false;
                    default: s += *p_; break;
                }
                ++p_;
            } else {
                s += *p_++;
            }
        }
        if (*p_ != '"') {
            return false;
        }
        ++p_;
        return true;
    }

    bool value(Value& v) {
        skip();
        char const c = *p_;
        if (c == '{') {
            v.kind = Value::Kind::Object;
            ++p_;
            skip();
            if (*p_ == '}') {
                ++p_;
                return true;
            }
            while (true) {
                skip();
                if (*p_ != '"') {
                    return false;
                }
                std::string key;
                if (!string_body(key)) {
                    return false;
                }
                skip();
                if (*p_ != ':') {
                    return false;
                }
                ++p_;
                Value member;
                if (!value(member)) {
                    return false;
                }
                v.object.emplace_back(std::move(key), std::move(member));
                skip();
                if (*p_ == ',') {
                    ++p_;
                    continue;
                }
                if (*p_ == '}') {
                    ++p_;
                    return true;
                }
                return false;
            }
        }
        if (c == '[') {
            v.kind = Value::Kind::Array;
            ++p_;
            skip();
            if (*p_ == ']') {
                ++p_;
                return true;
            }
            while (true) {
                Value element;
                if (!value(element)) {
                    return false;
                }
                v.array.push_back(std::move(element));
                skip();
                if (*p_ == ',') {
                    ++p_;
                    continue;
                }
                if (*p_ == ']') {
                    ++p_;
                    return true;
                }
                return false;
            }
        }
        if (c == '"') {
            v.kind = Value::Kind::String;
            return string_body(v.string);
        }
        if (literal("true")) {
            v.kind    = Value::Kind::Bool;
            v.boolean = true;
            return true;
        }
        if (literal("false")) {
            v.kind    = Value::Kind::Bool;
            v.boolean = false;
            return true;
        }
        if (literal("null")) {
            v.kind = Value::Kind::Null;
            return true;
        }
        char* end = nullptr;
        double const d = std::strtod(p_, &end);
        if (end == p_) {
            return false;
        }
        v.kind   = Value::Kind::Number;
        v.number = d;
        p_       = end;
        return true;
    }

    char const* p_;
};

inline bool parse(char const* text, Value& out) {
    if (!text) {
        return false;
    }
    Parser parser(text);
    return parser.parse(out);
}

inline double number_or(Value const* v, double fallback) {
    return (v && v->kind == Value::Kind::Number) ? v->number : fallback;
}

inline bool bool_or(Value const* v, bool fallback) {
    return (v && v->kind == Value::Kind::Bool) ? v->boolean : fallback;
}

inline std::string string_or(Value const* v, std::string const& fallback) {
    return (v && v->kind == Value::Kind::String) ? v->string : fallback;
}

// The value as JSON text (numbers with 17 significant digits), for handing a parsed
// sub-object to an entry point that takes a JSON string.
inline void dump(Value const& v, std::string& out) {
    switch (v.kind) {
        case Value::Kind::Null:
            out += "null";
            break;
        case Value::Kind::Bool:
            out += v.boolean ? "true" : "false";
            break;
        case Value::Kind::Number: {
            char buf[32];
            std::snprintf(buf, sizeof(buf), "%.17g", v.number);
            out += buf;
            break;
        }
        case Value::Kind::String:
            out += '"';
            for (char const c : v.string) {
                if (c == '"' || c == '\\') {
                    out += '\\';
                }
                out += c;
            }
            out += '"';
            break;
        case Value::Kind::Array:
            out += '[';
            for (size_t i = 0; i < v.array.size(); ++i) {
                out += i ? "," : "";
                dump(v.array[i], out);
            }
            out += ']';
            break;
        case Value::Kind::Object:
            out += '{';
            for (size_t i = 0; i < v.object.size(); ++i) {
                out += i ? "," : "";
                dump(Value{Value::Kind::String, false, 0.0, v.object[i].first, {}, {}}, out);
                out += ':';
                dump(v.object[i].second, out);
            }
            out += '}';
            break;
    }
}

inline std::string dump(Value const& v) {
    std::string out;
    dump(v, out);
    return out;
}

}  // namespace spb::json
