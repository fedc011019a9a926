#include "mas_json.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>

namespace pmas
{
    namespace
    {
        struct Parser
        {
            const std::string &s;
            size_t i = 0;
            explicit Parser(const std::string &t) : s(t) {}

            [[noreturn]] void fail(const char *what) const
            {
                throw std::runtime_error(std::string("json parse error: ") + what + " at offset " + std::to_string(i));
            }
            void ws()
            {
                while (i < s.size() && (s[i] == ' ' || s[i] == '\t' || s[i] == '\n' || s[i] == '\r'))
                    ++i;
            }
            bool lit(const char *w)
            {
                size_t n = 0;
                while (w[n])
                    ++n;
                if (s.compare(i, n, w) == 0)
                {
                    i += n;
                    return true;
                }
                return false;
            }
            std::string string_lit()
            {
                if (s[i] != '"')
                    fail("expected string");
                ++i;
                std::string out;
                while (i < s.size() && s[i] != '"')
                {
                    char c = s[i++];
                    if (c == '\\')
                    {
                        if (i >= s.size())
                            fail("bad escape");
                        char e = s[i++];
                        switch (e)
                        {
                        case '"':
                        case '\\':
                        case '/':
                            out += e;
                            break;
                        case 'b':
                            out += '\b';
                            break;
                        case 'f':
                            out += '\f';
                            break;
                        case 'n':
                            out += '\n';
                            break;
                        case 'r':
                            out += '\r';
                            break;
                        case 't':
                            out += '\t';
                            break;
                        case 'u':
                        {
                            if (i + 4 > s.size())
                                fail("bad unicode escape");
                            unsigned cp = (unsigned)std::strtoul(s.substr(i, 4).c_str(), nullptr, 16);
                            i += 4;
                            if (cp < 0x80)
                                out += (char)cp;
                            else if (cp < 0x800)
                            {
                                out += (char)(0xC0 | (cp >> 6));
                                out += (char)(0x80 | (cp & 0x3F));
                            }
                            else
                            {
                                out += (char)(0xE0 | (cp >> 12));
                                out += (char)(0x80 | ((cp >> 6) & 0x3F));
                                out += (char)(0x80 | (cp & 0x3F));
                            }
                            break;
                        }
                        default:
                            fail("bad escape");
                        }
                    }
                    else
                        out += c;
                }
                if (i >= s.size())
                    fail("unterminated string");
                ++i;
                return out;
            }
            Json value()
            {
                ws();
                if (i >= s.size())
                    fail("unexpected end");
                Json v;
                char c = s[i];
                if (c == '{')
                {
                    ++i;
                    v.type = Json::Object;
                    ws();
                    if (s[i] == '}')
                    {
                        ++i;
                        return v;
                    }
                    for (;;)
                    {
                        ws();
                        std::string k = string_lit();
                        ws();
                        if (i >= s.size() || s[i] != ':')
                            fail("expected ':'");
                        ++i;
                        Json item = value();
                        bool replaced = false;
                        for (auto &kv : v.obj)
                            if (kv.first == k)
                            {
                                kv.second = item;
                                replaced = true;
                            }
                        if (!replaced)
                            v.obj.emplace_back(k, item);
                        ws();
                        if (i < s.size() && s[i] == ',')
                        {
                            ++i;
                            continue;
                        }
                        if (i < s.size() && s[i] == '}')
                        {
                            ++i;
                            return v;
                        }
                        fail("expected ',' or '}'");
                    }
                }
                if (c == '[')
                {
                    ++i;
                    v.type = Json::Array;
                    ws();
                    if (s[i] == ']')
                    {
                        ++i;
                        return v;
                    }
                    for (;;)
                    {
                        v.arr.push_back(value());
                        ws();
                        if (i < s.size() && s[i] == ',')
                        {
                            ++i;
                            continue;
                        }
                        if (i < s.size() && s[i] == ']')
                        {
                            ++i;
                            return v;
                        }
                        fail("expected ',' or ']'");
                    }
                }
                if (c == '"')
                {
                    v.type = Json::String;
                    v.str = string_lit();
                    return v;
                }
                if (lit("true"))
                {
                    v.type = Json::Bool;
                    v.b = true;
                    return v;
                }
                if (lit("false"))
                {
                    v.type = Json::Bool;
                    v.b = false;
                    return v;
                }
                if (lit("null"))
                    return v;
                // number
                size_t start = i;
                if (s[i] == '-' || s[i] == '+')
                    ++i;
                bool integer = true;
                while (i < s.size() && (isdigit((unsigned char)s[i]) || s[i] == '.' || s[i] == 'e' || s[i] == 'E' ||
                                        s[i] == '-' || s[i] == '+'))
                {
                    if (s[i] == '.' || s[i] == 'e' || s[i] == 'E')
                        integer = false;
                    ++i;
                }
                if (start == i)
                    fail("unexpected character");
                std::string tok = s.substr(start, i - start);
                char *end = nullptr;
                double d = std::strtod(tok.c_str(), &end);
                if (!end || *end != '\0')
                    fail("bad number");
                v.type = Json::Number;
                v.num = d;
                v.is_integer = integer;
                return v;
            }
        };

        void dump_string(const std::string &s, std::string &out)
        {
            out += '"';
            for (char c : s)
            {
                switch (c)
                {
                case '"':
                    out += "\\\"";
                    break;
                case '\\':
                    out += "\\\\";
                    break;
                case '\n':
                    out += "\\n";
                    break;
                case '\t':
                    out += "\\t";
                    break;
                default:
                    out += c;
                }
            }
            out += '"';
        }

        void dump_value(const Json &v, std::string &out)
        {
            char buf[64];
            switch (v.type)
            {
            case Json::Null:
                out += "null";
                break;
            case Json::Bool:
                out += v.b ? "true" : "false";
                break;
            case Json::Number:
                if (!std::isfinite(v.num))
                {
                    out += "null"; // JSON has no NaN / infinity
                    break;
                }
                if (v.is_integer && std::fabs(v.num) < 9e15)
                    std::snprintf(buf, sizeof(buf), "%lld", (long long)v.num);
                else
                    std::snprintf(buf, sizeof(buf), "%.17g", v.num);
                out += buf;
                break;
            case Json::String:
                dump_string(v.str, out);
                break;
            case Json::Array:
                out += '[';
                for (size_t k = 0; k < v.arr.size(); ++k)
                {
                    if (k)
                        out += ',';
                    dump_value(v.arr[k], out);
                }
                out += ']';
                break;
            case Json::Object:
                out += '{';
                for (size_t k = 0; k < v.obj.size(); ++k)
                {
                    if (k)
                        out += ',';
                    dump_string(v.obj[k].first, out);
                    out += ':';
                    dump_value(v.obj[k].second, out);
                }
                out += '}';
                break;
            }
        }
    } // namespace

    const Json *Json::find(const std::string &key) const
    {
        if (type != Object)
            return nullptr;
        for (const auto &kv : obj)
            if (kv.first == key)
                return &kv.second;
        return nullptr;
    }

    Json Json::parse(const std::string &text)
    {
        Parser p(text);
        Json v = p.value();
        p.ws();
        if (p.i != text.size())
            p.fail("trailing characters");
        return v;
    }

    std::string Json::dump() const
    {
        std::string out;
        dump_value(*this, out);
        return out;
    }
} // namespace pmas
