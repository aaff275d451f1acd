// Plan files: a reader for the libconfig text format the reference's plans
// use (README.md:66-170, drivers/sample_queries/q1/query1.conf):
//   name = value;  name : value;  groups { ... }, lists ( ... ),
//   arrays [ ... ], strings "...", integers, floats, booleans, and
//   #, // and /* */ comments.
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace pyg_host {

struct PlanError : std::runtime_error {
    explicit PlanError(const std::string& m) : std::runtime_error(m) {}
};

class Setting {
public:
    enum Type { Group, List, Array, Int, Float, String, Bool };

    Type type = Group;
    std::string name;
    int64_t i = 0;
    double f = 0;
    std::string s;
    bool b = false;
    std::vector<std::unique_ptr<Setting>> items;  // group members / list and array elements

    bool exists(const std::string& key) const;
    const Setting& operator[](const std::string& key) const;
    const Setting& operator[](size_t idx) const;
    size_t size() const { return items.size(); }
    bool isAggregate() const { return type == Group || type == List || type == Array; }
    bool isNumber() const { return type == Int || type == Float; }

    int64_t asInt() const;
    double asFloat() const;
    const std::string& asString() const;
    // Integer member with a default when absent.
    int64_t getInt(const std::string& key, int64_t dflt) const;
    std::string getString(const std::string& key, const std::string& dflt) const;
};

// Parses a whole plan; the root is a group.
std::unique_ptr<Setting> parse_plan(const std::string& text);
std::unique_ptr<Setting> parse_plan_file(const std::string& path);

}  // namespace pyg_host
