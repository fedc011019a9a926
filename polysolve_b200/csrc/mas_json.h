// Minimal JSON value + parser for solver parameters (objects, arrays, strings, numbers, bools,
// null). polysolve passes parameters as nlohmann::json; across the C ABI they travel as text.
#pragma once

#include <map>
#include <memory>
#include <string>
#include <vector>

namespace pmas
{
    struct Json
    {
        enum Type
        {
            Null,
            Bool,
            Number,
            String,
            Array,
            Object
        } type = Null;
        bool b = false;
        double num = 0.0;
        bool is_integer = false;
        std::string str;
        std::vector<Json> arr;
        std::vector<std::pair<std::string, Json>> obj; // insertion order kept

        const Json *find(const std::string &key) const;
        bool contains(const std::string &key) const { return find(key) != nullptr; }
        static Json parse(const std::string &text); // throws std::runtime_error
        std::string dump() const;
    };
} // namespace pmas
