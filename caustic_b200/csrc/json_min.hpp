// Minimal JSON reader for the solver's parameter file.
//
// Plays the role of the reference's JsonHandler (Optimal_Transport_rl/
// ConfigLoader.h:13-89, over nlohmann::json, which is not available here):
// load a file, read typed values, arrays and nested objects, and throw
// std::runtime_error naming the key when it is missing or of the wrong type.
#pragma once
#include <cctype>
#include <cstdlib>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace jmin {

struct Value {
    enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::vector<Value> arr;
    std::map<std::string, Value> obj;
};

class Parser {
public:
    explicit Parser(const std::string &t) : s_(t) {}
    Value parse()
    {
        Value v = value();
        ws();
        if (i_ != s_.size()) fail("trailing characters");
        return v;
    }

private:
    const std::string &s_;
    size_t i_ = 0;

    [[noreturn]] void fail(const std::string &m) const
    {
        throw std::runtime_error("JSON parse error at offset " + std::to_string(i_) + ": " + m);
    }
    void ws()
    {
        while (i_ < s_.size() && std::isspace((unsigned char)s_[i_])) i_++;
    }
    bool take(char c)
    {
        ws();
        if (i_ < s_.size() && s_[i_] == c) {
            i_++;
            return true;
        }
        return false;
    }
    void expect(char c)
    {
        if (!take(c)) fail(std::string("expected '") + c + "'");
    }
    Value value()
    {
        ws();
        if (i_ >= s_.size()) fail("unexpected end");
        char c = s_[i_];
        Value v;
        if (c == '{') {
            i_++;
            v.kind = Value::Object;
            if (take('}')) return v;
            do {
                ws();
                std::string k = string_lit();
                expect(':');
                v.obj[k] = value();
            } while (take(','));
            expect('}');
        } else if (c == '[') {
            i_++;
            v.kind = Value::Array;
            if (take(']')) return v;
            do {
                v.arr.push_back(value());
            } while (take(','));
            expect(']');
        } else if (c == '"') {
            v.kind = Value::String;
            v.str = string_lit();
        } else if (s_.compare(i_, 4, "true") == 0) {
            i_ += 4;
            v.kind = Value::Bool;
            v.b = true;
        } else if (s_.compare(i_, 5, "false") == 0) {
            i_ += 5;
            v.kind = Value::Bool;
        } else if (s_.compare(i_, 4, "null") == 0) {
            i_ += 4;
        } else {
            const char *b = s_.c_str() + i_;
            char *e = nullptr;
            v.num = std::strtod(b, &e);
            if (e == b) fail("bad value");
            i_ += (size_t)(e - b);
            v.kind = Value::Number;
        }
        return v;
    }
    std::string string_lit()
    {
        if (i_ >= s_.size() || s_[i_] != '"') fail("expected string");
        i_++;
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
                    // keep the code point as UTF-8 (comments may be non-ASCII)
                    if (i_ + 4 > s_.size()) fail("bad \\u escape");
                    unsigned cp = (unsigned)std::stoul(s_.substr(i_, 4), nullptr, 16);
                    i_ += 4;
                    if (cp < 0x80) out += (char)cp;
                    else if (cp < 0x800) { out += (char)(0xC0 | (cp >> 6)); out += (char)(0x80 | (cp & 0x3F)); }
                    else { out += (char)(0xE0 | (cp >> 12)); out += (char)(0x80 | ((cp >> 6) & 0x3F)); out += (char)(0x80 | (cp & 0x3F)); }
                    break;
                }
                default: out += e; break;
                }
            } else {
                out += c;
            }
        }
        if (i_ >= s_.size()) fail("unterminated string");
        i_++;
        return out;
    }
};

// JsonHandler-like view: getValue / getArray / getObject with key errors.
class Handler {
public:
    Handler() = default;
    explicit Handler(Value v) : v_(std::make_shared<Value>(std::move(v))) {}

    bool loadFromFile(const std::string &path, std::string *err = nullptr)
    {
        std::ifstream f(path);
        if (!f) {
            if (err) *err = "Failed to open JSON file: " + path;
            return false;
        }
        std::stringstream ss;
        ss << f.rdbuf();
        try {
            v_ = std::make_shared<Value>(Parser(ss.str()).parse());
        } catch (const std::exception &e) {
            if (err) *err = e.what();
            return false;
        }
        if (v_->kind != Value::Object) {
            if (err) *err = "JSON root is not an object";
            return false;
        }
        return true;
    }

    const Value &at(const std::string &k) const
    {
        if (!v_ || v_->kind != Value::Object) throw std::runtime_error("not an object");
        auto it = v_->obj.find(k);
        if (it == v_->obj.end()) throw std::runtime_error("Key does not exist: " + k);
        return it->second;
    }
    bool has(const std::string &k) const { return v_ && v_->obj.count(k) > 0; }

    double number(const std::string &k) const
    {
        const Value &v = at(k);
        if (v.kind != Value::Number) throw std::runtime_error("Type error for key '" + k + "': not a number");
        return v.num;
    }
    int integer(const std::string &k) const { return (int)number(k); }
    bool boolean(const std::string &k) const
    {
        const Value &v = at(k);
        if (v.kind != Value::Bool) throw std::runtime_error("Type error for key '" + k + "': not a bool");
        return v.b;
    }
    std::string string(const std::string &k) const
    {
        const Value &v = at(k);
        if (v.kind != Value::String) throw std::runtime_error("Type error for key '" + k + "': not a string");
        return v.str;
    }
    std::vector<double> numbers(const std::string &k) const
    {
        const Value &v = at(k);
        if (v.kind != Value::Array) throw std::runtime_error("Invalid array key: " + k);
        std::vector<double> out;
        for (const Value &e : v.arr) {
            if (e.kind != Value::Number) throw std::runtime_error("Array type error for key '" + k + "'");
            out.push_back(e.num);
        }
        return out;
    }
    Handler object(const std::string &k) const
    {
        const Value &v = at(k);
        if (v.kind != Value::Object) throw std::runtime_error("Key '" + k + "' is not a JSON object");
        return Handler(v);
    }

private:
    std::shared_ptr<Value> v_;
};

}  // namespace jmin
