// A read-only JSON document with the yyjson API subset that the reference's
// Blender scene bundle importer calls (src/adapter/blender_scene*.cpp,
// src/adapter/blender_graph_*.cpp).  Test infrastructure: yyjson itself is
// vendored only by the reference's LuisaCompute submodule, which is empty in
// this checkout, so the importer is compiled here against this header.  A
// maintainer who links the importer with the CUDA backend uses the real
// yyjson; nothing here is part of libpsycles_cuda.so.
//
// Semantics follow yyjson's published reader with no flags (RFC 8259 JSON,
// no comments, no trailing commas, no NaN/Inf literals):
// - an integer literal without fraction or exponent is an unsigned integer
//   when non-negative and a signed integer when negative; one that does not
//   fit in 64 bits is read as a real;
// - every other number is a real (correctly rounded, as strtod does);
// - strings are UTF-8 with escapes decoded (\uXXXX surrogate pairs joined);
// - object lookups return the first member with the key;
// - every accessor accepts a null value and answers false, 0 or nullptr.
#pragma once

#include <cerrno>
#include <clocale>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <locale.h>
#include <string>
#include <utility>
#include <vector>

enum yyjson_shim_tag : uint8_t {
    YYJSON_SHIM_NULL,
    YYJSON_SHIM_BOOL,
    YYJSON_SHIM_UINT,
    YYJSON_SHIM_SINT,
    YYJSON_SHIM_REAL,
    YYJSON_SHIM_STR,
    YYJSON_SHIM_ARR,
    YYJSON_SHIM_OBJ,
};

struct yyjson_val {
    yyjson_shim_tag tag = YYJSON_SHIM_NULL;
    bool boolean = false;
    uint64_t uint_value = 0;
    int64_t sint_value = 0;
    double real = 0.0;
    std::string str;
    std::vector<yyjson_val *> items;                            // array elements
    std::vector<std::pair<std::string, yyjson_val *>> members;  // object members, in order
};

struct yyjson_doc {
    std::deque<yyjson_val> values;  // stable addresses
    yyjson_val *root = nullptr;
};

typedef uint32_t yyjson_read_flag;
typedef uint32_t yyjson_read_code;
struct yyjson_alc;

struct yyjson_read_err {
    yyjson_read_code code;
    const char *msg;
    size_t pos;
};

struct yyjson_arr_iter {
    size_t idx;
    size_t max;
    yyjson_val *cur;
    yyjson_val *arr;
};

namespace yyjson_shim {

class Parser {
public:
    Parser(const char *text, size_t size, yyjson_doc *doc) : p_(text), begin_(text), end_(text + size), doc_(doc) {}

    bool parse(const char **message, size_t *pos) {
        skip_space();
        yyjson_val *root = value(0);
        if (root) {
            skip_space();
            if (p_ != end_) fail("unexpected content after document");
        }
        if (error_) {
            *message = error_;
            *pos = size_t(p_ - begin_);
            return false;
        }
        doc_->root = root;
        return true;
    }

private:
    const char *p_;
    const char *begin_;
    const char *end_;
    yyjson_doc *doc_;
    const char *error_ = nullptr;

    yyjson_val *fail(const char *message) {
        if (!error_) error_ = message;
        return nullptr;
    }
    yyjson_val *make(yyjson_shim_tag tag) {
        doc_->values.emplace_back();
        doc_->values.back().tag = tag;
        return &doc_->values.back();
    }
    void skip_space() {
        while (p_ != end_ && (*p_ == ' ' || *p_ == '\t' || *p_ == '\n' || *p_ == '\r')) ++p_;
    }
    bool literal(const char *word) {
        const size_t n = std::strlen(word);
        if (size_t(end_ - p_) < n || std::memcmp(p_, word, n) != 0) return false;
        p_ += n;
        return true;
    }

    yyjson_val *value(int depth) {
        if (depth > 1024) return fail("document nested too deeply");
        if (p_ == end_) return fail("unexpected end of data");
        switch (*p_) {
            case '{': return object(depth);
            case '[': return array(depth);
            case '"': {
                yyjson_val *v = make(YYJSON_SHIM_STR);
                if (!string(&v->str)) return nullptr;
                return v;
            }
            case 't':
                if (literal("true")) {
                    yyjson_val *v = make(YYJSON_SHIM_BOOL);
                    v->boolean = true;
                    return v;
                }
                return fail("invalid literal");
            case 'f':
                if (literal("false")) return make(YYJSON_SHIM_BOOL);
                return fail("invalid literal");
            case 'n':
                if (literal("null")) return make(YYJSON_SHIM_NULL);
                return fail("invalid literal");
            default: return number();
        }
    }

    yyjson_val *object(int depth) {
        yyjson_val *v = make(YYJSON_SHIM_OBJ);
        ++p_;
        skip_space();
        if (p_ != end_ && *p_ == '}') {
            ++p_;
            return v;
        }
        for (;;) {
            skip_space();
            if (p_ == end_ || *p_ != '"') return fail("object key is not a string");
            std::string key;
            if (!string(&key)) return nullptr;
            skip_space();
            if (p_ == end_ || *p_ != ':') return fail("missing colon after object key");
            ++p_;
            skip_space();
            yyjson_val *member = value(depth + 1);
            if (!member) return nullptr;
            v->members.emplace_back(std::move(key), member);
            skip_space();
            if (p_ == end_) return fail("unexpected end of data");
            if (*p_ == ',') {
                ++p_;
                continue;
            }
            if (*p_ == '}') {
                ++p_;
                return v;
            }
            return fail("unexpected character in object");
        }
    }

    yyjson_val *array(int depth) {
        yyjson_val *v = make(YYJSON_SHIM_ARR);
        ++p_;
        skip_space();
        if (p_ != end_ && *p_ == ']') {
            ++p_;
            return v;
        }
        for (;;) {
            skip_space();
            yyjson_val *item = value(depth + 1);
            if (!item) return nullptr;
            v->items.push_back(item);
            skip_space();
            if (p_ == end_) return fail("unexpected end of data");
            if (*p_ == ',') {
                ++p_;
                continue;
            }
            if (*p_ == ']') {
                ++p_;
                return v;
            }
            return fail("unexpected character in array");
        }
    }

    static void append_utf8(std::string *out, uint32_t cp) {
        if (cp < 0x80u) {
            out->push_back(char(cp));
        } else if (cp < 0x800u) {
            out->push_back(char(0xC0u | (cp >> 6)));
            out->push_back(char(0x80u | (cp & 0x3Fu)));
        } else if (cp < 0x10000u) {
            out->push_back(char(0xE0u | (cp >> 12)));
            out->push_back(char(0x80u | ((cp >> 6) & 0x3Fu)));
            out->push_back(char(0x80u | (cp & 0x3Fu)));
        } else {
            out->push_back(char(0xF0u | (cp >> 18)));
            out->push_back(char(0x80u | ((cp >> 12) & 0x3Fu)));
            out->push_back(char(0x80u | ((cp >> 6) & 0x3Fu)));
            out->push_back(char(0x80u | (cp & 0x3Fu)));
        }
    }

    bool hex4(uint32_t *out) {
        if (end_ - p_ < 4) return false;
        uint32_t v = 0;
        for (int i = 0; i < 4; ++i) {
            const char c = p_[i];
            v <<= 4;
            if (c >= '0' && c <= '9') v |= uint32_t(c - '0');
            else if (c >= 'a' && c <= 'f') v |= uint32_t(c - 'a' + 10);
            else if (c >= 'A' && c <= 'F') v |= uint32_t(c - 'A' + 10);
            else return false;
        }
        p_ += 4;
        *out = v;
        return true;
    }

    bool string(std::string *out) {
        ++p_;  // opening quote
        for (;;) {
            if (p_ == end_) {
                fail("unclosed string");
                return false;
            }
            const unsigned char c = static_cast<unsigned char>(*p_);
            if (c == '"') {
                ++p_;
                return true;
            }
            if (c < 0x20u) {
                fail("unexpected control character in string");
                return false;
            }
            if (c != '\\') {
                out->push_back(char(c));
                ++p_;
                continue;
            }
            ++p_;
            if (p_ == end_) {
                fail("unclosed string");
                return false;
            }
            const char e = *p_++;
            switch (e) {
                case '"': out->push_back('"'); break;
                case '\\': out->push_back('\\'); break;
                case '/': out->push_back('/'); break;
                case 'b': out->push_back('\b'); break;
                case 'f': out->push_back('\f'); break;
                case 'n': out->push_back('\n'); break;
                case 'r': out->push_back('\r'); break;
                case 't': out->push_back('\t'); break;
                case 'u': {
                    uint32_t cp = 0;
                    if (!hex4(&cp)) {
                        fail("invalid escaped unicode in string");
                        return false;
                    }
                    if (cp >= 0xD800u && cp <= 0xDBFFu) {
                        uint32_t low = 0;
                        if (end_ - p_ < 2 || p_[0] != '\\' || p_[1] != 'u') {
                            fail("no low surrogate in string");
                            return false;
                        }
                        p_ += 2;
                        if (!hex4(&low) || low < 0xDC00u || low > 0xDFFFu) {
                            fail("invalid low surrogate in string");
                            return false;
                        }
                        cp = 0x10000u + ((cp - 0xD800u) << 10) + (low - 0xDC00u);
                    } else if (cp >= 0xDC00u && cp <= 0xDFFFu) {
                        fail("no high surrogate in string");
                        return false;
                    }
                    append_utf8(out, cp);
                    break;
                }
                default: fail("invalid escaped character in string"); return false;
            }
        }
    }

    yyjson_val *number() {
        const char *start = p_;
        bool negative = false;
        if (p_ != end_ && *p_ == '-') {
            negative = true;
            ++p_;
        }
        if (p_ == end_ || *p_ < '0' || *p_ > '9') return fail("invalid number");
        if (*p_ == '0') {
            ++p_;
            if (p_ != end_ && *p_ >= '0' && *p_ <= '9') return fail("number with leading zero");
        } else {
            while (p_ != end_ && *p_ >= '0' && *p_ <= '9') ++p_;
        }
        bool integral = true;
        if (p_ != end_ && *p_ == '.') {
            integral = false;
            ++p_;
            if (p_ == end_ || *p_ < '0' || *p_ > '9') return fail("no digit after decimal point");
            while (p_ != end_ && *p_ >= '0' && *p_ <= '9') ++p_;
        }
        if (p_ != end_ && (*p_ == 'e' || *p_ == 'E')) {
            integral = false;
            ++p_;
            if (p_ != end_ && (*p_ == '+' || *p_ == '-')) ++p_;
            if (p_ == end_ || *p_ < '0' || *p_ > '9') return fail("no digit after exponent sign");
            while (p_ != end_ && *p_ >= '0' && *p_ <= '9') ++p_;
        }
        const std::string literal_text(start, p_);
        if (integral) {
            // digits only (and a leading minus): accumulate with overflow check
            const char *d = literal_text.c_str() + (negative ? 1 : 0);
            uint64_t magnitude = 0;
            bool overflow = false;
            for (; *d; ++d) {
                const uint64_t digit = uint64_t(*d - '0');
                if (magnitude > (UINT64_MAX - digit) / 10u) {
                    overflow = true;
                    break;
                }
                magnitude = magnitude * 10u + digit;
            }
            if (!overflow && !negative) {
                yyjson_val *v = make(YYJSON_SHIM_UINT);
                v->uint_value = magnitude;
                return v;
            }
            if (!overflow && negative && magnitude <= uint64_t(INT64_MAX) + 1u) {
                yyjson_val *v = make(YYJSON_SHIM_SINT);
                v->sint_value = magnitude == uint64_t(INT64_MAX) + 1u ? INT64_MIN : -int64_t(magnitude);
                return v;
            }
        }
        // JSON numbers use '.', whatever the C locale says
        locale_t c_locale = newlocale(LC_NUMERIC_MASK, "C", locale_t(0));
        const double real = strtod_l(literal_text.c_str(), nullptr, c_locale);
        freelocale(c_locale);
        if (real == HUGE_VAL || real == -HUGE_VAL) return fail("number is infinity when parsed as double");
        yyjson_val *v = make(YYJSON_SHIM_REAL);
        v->real = real;
        return v;
    }
};

}  // namespace yyjson_shim

inline yyjson_doc *yyjson_read_opts(const char *text, size_t size, yyjson_read_err *err) {
    yyjson_doc *doc = new yyjson_doc();
    const char *message = nullptr;
    size_t pos = 0;
    yyjson_shim::Parser parser(text, size, doc);
    if (!parser.parse(&message, &pos)) {
        delete doc;
        if (err) *err = yyjson_read_err{1u, message, pos};
        return nullptr;
    }
    if (err) *err = yyjson_read_err{0u, nullptr, 0u};
    return doc;
}

inline yyjson_doc *yyjson_read_file(const char *path, yyjson_read_flag, const yyjson_alc *, yyjson_read_err *err) {
    std::FILE *file = path ? std::fopen(path, "rb") : nullptr;
    if (!file) {
        if (err) *err = yyjson_read_err{2u, "file opening failed", 0u};
        return nullptr;
    }
    std::string text;
    char chunk[65536];
    size_t n = 0;
    while ((n = std::fread(chunk, 1, sizeof(chunk), file)) > 0) text.append(chunk, n);
    const bool read_error = std::ferror(file) != 0;
    std::fclose(file);
    if (read_error) {
        if (err) *err = yyjson_read_err{3u, "file reading failed", 0u};
        return nullptr;
    }
    if (text.empty()) {
        if (err) *err = yyjson_read_err{4u, "input data is empty", 0u};
        return nullptr;
    }
    return yyjson_read_opts(text.data(), text.size(), err);
}

inline void yyjson_doc_free(yyjson_doc *doc) { delete doc; }
inline yyjson_val *yyjson_doc_get_root(yyjson_doc *doc) { return doc ? doc->root : nullptr; }

inline bool yyjson_is_null(yyjson_val *v) { return v && v->tag == YYJSON_SHIM_NULL; }
inline bool yyjson_is_bool(yyjson_val *v) { return v && v->tag == YYJSON_SHIM_BOOL; }
inline bool yyjson_is_uint(yyjson_val *v) { return v && v->tag == YYJSON_SHIM_UINT; }
inline bool yyjson_is_sint(yyjson_val *v) { return v && v->tag == YYJSON_SHIM_SINT; }
inline bool yyjson_is_int(yyjson_val *v) { return yyjson_is_uint(v) || yyjson_is_sint(v); }
inline bool yyjson_is_real(yyjson_val *v) { return v && v->tag == YYJSON_SHIM_REAL; }
inline bool yyjson_is_num(yyjson_val *v) { return yyjson_is_int(v) || yyjson_is_real(v); }
inline bool yyjson_is_str(yyjson_val *v) { return v && v->tag == YYJSON_SHIM_STR; }
inline bool yyjson_is_arr(yyjson_val *v) { return v && v->tag == YYJSON_SHIM_ARR; }
inline bool yyjson_is_obj(yyjson_val *v) { return v && v->tag == YYJSON_SHIM_OBJ; }

inline bool yyjson_get_bool(yyjson_val *v) { return yyjson_is_bool(v) && v->boolean; }
inline uint64_t yyjson_get_uint(yyjson_val *v) {
    if (yyjson_is_uint(v)) return v->uint_value;
    if (yyjson_is_sint(v)) return uint64_t(v->sint_value);
    return 0u;
}
inline int64_t yyjson_get_sint(yyjson_val *v) {
    if (yyjson_is_sint(v)) return v->sint_value;
    if (yyjson_is_uint(v)) return int64_t(v->uint_value);
    return 0;
}
inline double yyjson_get_real(yyjson_val *v) { return yyjson_is_real(v) ? v->real : 0.0; }
inline double yyjson_get_num(yyjson_val *v) {
    if (yyjson_is_real(v)) return v->real;
    if (yyjson_is_uint(v)) return double(v->uint_value);
    if (yyjson_is_sint(v)) return double(v->sint_value);
    return 0.0;
}
inline const char *yyjson_get_str(yyjson_val *v) { return yyjson_is_str(v) ? v->str.c_str() : nullptr; }

inline size_t yyjson_arr_size(yyjson_val *v) { return yyjson_is_arr(v) ? v->items.size() : 0u; }
inline yyjson_val *yyjson_arr_get(yyjson_val *v, size_t idx) {
    return yyjson_is_arr(v) && idx < v->items.size() ? v->items[idx] : nullptr;
}
inline yyjson_arr_iter yyjson_arr_iter_with(yyjson_val *v) {
    yyjson_arr_iter iter{0u, yyjson_arr_size(v), nullptr, yyjson_is_arr(v) ? v : nullptr};
    return iter;
}
inline bool yyjson_arr_iter_init(yyjson_val *v, yyjson_arr_iter *iter) {
    if (!iter) return false;
    *iter = yyjson_arr_iter_with(v);
    return iter->arr != nullptr;
}
inline bool yyjson_arr_iter_has_next(yyjson_arr_iter *iter) { return iter && iter->idx < iter->max; }
inline yyjson_val *yyjson_arr_iter_next(yyjson_arr_iter *iter) {
    if (!iter || !iter->arr || iter->idx >= iter->max) return nullptr;
    iter->cur = iter->arr->items[iter->idx++];
    return iter->cur;
}

inline size_t yyjson_obj_size(yyjson_val *v) { return yyjson_is_obj(v) ? v->members.size() : 0u; }
inline yyjson_val *yyjson_obj_get(yyjson_val *v, const char *key) {
    if (!yyjson_is_obj(v) || !key) return nullptr;
    for (auto &member : v->members)
        if (member.first == key) return member.second;
    return nullptr;
}
