// Tiny JSON reader exposing the subset of the nlohmann::json interface that
// the reference's SceneParameter.h uses: parse(stream), at(key), operator[](i),
// size(), range-for over arrays and get<T>() for numbers, bools, strings and
// vectors of numbers.  TEST INFRASTRUCTURE (reference cross-check build only).
#pragma once
#include <cctype>
#include <istream>
#include <iterator>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

namespace nlohmann {

class json {
public:
    enum class Kind { Null, Bool, Number, String, Array, Object };
    Kind kind = Kind::Null;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::vector<json> arr;
    std::vector<std::pair<std::string, json>> obj;

    template <typename Stream> static json parse(Stream&& in) {
        std::string text((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
        size_t pos = 0;
        json j = parse_value(text, pos);
        return j;
    }

    const json& at(const std::string& key) const {
        if (kind != Kind::Object) throw std::out_of_range("json: not an object");
        for (const auto& kv : obj)
            if (kv.first == key) return kv.second;
        throw std::out_of_range("json: missing key " + key);
    }
    const json& at(size_t i) const {
        if (kind != Kind::Array || i >= arr.size()) throw std::out_of_range("json: bad index");
        return arr[i];
    }
    const json& operator[](size_t i) const { return at(i); }
    size_t size() const { return kind == Kind::Array ? arr.size() : (kind == Kind::Object ? obj.size() : 0); }
    std::vector<json>::const_iterator begin() const { return arr.begin(); }
    std::vector<json>::const_iterator end() const { return arr.end(); }

    template <typename T> T get() const { return getter<T>::run(*this); }

private:
    template <typename T, typename = void> struct getter;
    template <typename T> struct getter<T, std::enable_if_t<std::is_arithmetic<T>::value && !std::is_same<T, bool>::value>> {
        static T run(const json& j) {
            if (j.kind == Kind::Bool) return T(j.b);
            if (j.kind != Kind::Number) throw std::runtime_error("json: not a number");
            return static_cast<T>(j.num);
        }
    };
    template <typename T> struct getter<T, std::enable_if_t<std::is_same<T, bool>::value>> {
        static T run(const json& j) {
            if (j.kind != Kind::Bool) throw std::runtime_error("json: not a bool");
            return j.b;
        }
    };
    template <typename T> struct getter<T, std::enable_if_t<std::is_same<T, std::string>::value>> {
        static T run(const json& j) {
            if (j.kind != Kind::String) throw std::runtime_error("json: not a string");
            return j.str;
        }
    };
    template <typename E> struct getter<std::vector<E>, void> {
        static std::vector<E> run(const json& j) {
            std::vector<E> out;
            for (const auto& e : j.arr) out.push_back(e.template get<E>());
            return out;
        }
    };

    static void skip(const std::string& t, size_t& p) {
        while (p < t.size() && std::isspace(static_cast<unsigned char>(t[p]))) ++p;
    }
    static json parse_value(const std::string& t, size_t& p) {
        skip(t, p);
        if (p >= t.size()) throw std::runtime_error("json: unexpected end");
        json j;
        char c = t[p];
        if (c == '{') {
            j.kind = Kind::Object;
            ++p;
            skip(t, p);
            if (t[p] == '}') {
                ++p;
                return j;
            }
            while (true) {
                skip(t, p);
                json key = parse_value(t, p);
                skip(t, p);
                if (t[p] != ':') throw std::runtime_error("json: expected ':'");
                ++p;
                json val = parse_value(t, p);
                j.obj.emplace_back(key.str, val);
                skip(t, p);
                if (t[p] == ',') {
                    ++p;
                    continue;
                }
                if (t[p] == '}') {
                    ++p;
                    break;
                }
                throw std::runtime_error("json: expected ',' or '}'");
            }
        } else if (c == '[') {
            j.kind = Kind::Array;
            ++p;
            skip(t, p);
            if (t[p] == ']') {
                ++p;
                return j;
            }
            while (true) {
                j.arr.push_back(parse_value(t, p));
                skip(t, p);
                if (t[p] == ',') {
                    ++p;
                    continue;
                }
                if (t[p] == ']') {
                    ++p;
                    break;
                }
                throw std::runtime_error("json: expected ',' or ']'");
            }
        } else if (c == '"') {
            j.kind = Kind::String;
            ++p;
            while (p < t.size() && t[p] != '"') {
                if (t[p] == '\\' && p + 1 < t.size()) ++p;
                j.str.push_back(t[p++]);
            }
            ++p;
        } else if (t.compare(p, 4, "true") == 0) {
            j.kind = Kind::Bool;
            j.b = true;
            p += 4;
        } else if (t.compare(p, 5, "false") == 0) {
            j.kind = Kind::Bool;
            j.b = false;
            p += 5;
        } else if (t.compare(p, 4, "null") == 0) {
            p += 4;
        } else {
            size_t q = p;
            while (q < t.size() && (std::isdigit(static_cast<unsigned char>(t[q])) || t[q] == '-' || t[q] == '+' ||
                                    t[q] == '.' || t[q] == 'e' || t[q] == 'E'))
                ++q;
            j.kind = Kind::Number;
            j.num = std::stod(t.substr(p, q - p));
            p = q;
        }
        return j;
    }
};

}  // namespace nlohmann
