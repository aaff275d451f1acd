// Plan file reader (libconfig text format subset used by the reference's
// plans).  A recursive-descent parser over a character cursor.
#include "plan.h"

#include <cctype>
#include <cstdlib>
#include <fstream>
#include <sstream>

namespace pyg_host {

bool Setting::exists(const std::string& key) const
{
    if (type != Group) return false;
    for (auto& c : items)
        if (c->name == key) return true;
    return false;
}

const Setting& Setting::operator[](const std::string& key) const
{
    if (type == Group)
        for (auto& c : items)
            if (c->name == key) return *c;
    throw PlanError("missing setting '" + key + "'" + (name.empty() ? "" : " in '" + name + "'"));
}

const Setting& Setting::operator[](size_t idx) const
{
    if (idx >= items.size()) throw PlanError("index " + std::to_string(idx) + " out of range in '" + name + "'");
    return *items[idx];
}

int64_t Setting::asInt() const
{
    if (type == Int) return i;
    if (type == Float) return (int64_t)f;
    if (type == Bool) return b ? 1 : 0;
    throw PlanError("setting '" + name + "' is not a number");
}

double Setting::asFloat() const
{
    if (type == Float) return f;
    if (type == Int) return (double)i;
    throw PlanError("setting '" + name + "' is not a number");
}

const std::string& Setting::asString() const
{
    if (type != String) throw PlanError("setting '" + name + "' is not a string");
    return s;
}

int64_t Setting::getInt(const std::string& key, int64_t dflt) const { return exists(key) ? (*this)[key].asInt() : dflt; }

std::string Setting::getString(const std::string& key, const std::string& dflt) const
{
    return exists(key) ? (*this)[key].asString() : dflt;
}

namespace {

struct Parser {
    const std::string& t;
    size_t p = 0;
    int line = 1;

    explicit Parser(const std::string& text) : t(text) {}

    [[noreturn]] void fail(const std::string& m) const
    {
        throw PlanError("plan parse error at line " + std::to_string(line) + ": " + m);
    }

    void skip()
    {
        for (;;) {
            while (p < t.size() && isspace((unsigned char)t[p])) {
                if (t[p] == '\n') ++line;
                ++p;
            }
            if (p < t.size() && t[p] == '#') {
                while (p < t.size() && t[p] != '\n') ++p;
            } else if (p + 1 < t.size() && t[p] == '/' && t[p + 1] == '/') {
                while (p < t.size() && t[p] != '\n') ++p;
            } else if (p + 1 < t.size() && t[p] == '/' && t[p + 1] == '*') {
                size_t e = t.find("*/", p + 2);
                if (e == std::string::npos) fail("unterminated comment");
                for (size_t k = p; k < e; ++k)
                    if (t[k] == '\n') ++line;
                p = e + 2;
            } else {
                return;
            }
        }
    }

    bool peek(char c)
    {
        skip();
        return p < t.size() && t[p] == c;
    }

    void expect(char c)
    {
        if (!peek(c)) fail(std::string("expected '") + c + "'");
        ++p;
    }

    std::string ident()
    {
        skip();
        size_t s = p;
        while (p < t.size() && (isalnum((unsigned char)t[p]) || t[p] == '_' || t[p] == '-' || t[p] == '*')) ++p;
        if (s == p) fail("expected a setting name");
        return t.substr(s, p - s);
    }

    std::unique_ptr<Setting> value()
    {
        skip();
        if (p >= t.size()) fail("unexpected end of plan");
        auto v = std::make_unique<Setting>();
        char c = t[p];
        if (c == '{') {
            ++p;
            v->type = Setting::Group;
            while (!peek('}')) v->items.push_back(setting());
            ++p;
        } else if (c == '(' || c == '[') {
            char close = c == '(' ? ')' : ']';
            v->type = c == '(' ? Setting::List : Setting::Array;
            ++p;
            while (!peek(close)) {
                v->items.push_back(value());
                if (peek(',')) ++p;
            }
            ++p;
        } else if (c == '"') {
            v->type = Setting::String;
            while (peek('"')) {  // adjacent strings concatenate
                ++p;
                while (p < t.size() && t[p] != '"') {
                    if (t[p] == '\\' && p + 1 < t.size()) {
                        ++p;
                        char e = t[p];
                        v->s += e == 'n' ? '\n' : e == 't' ? '\t' : e;
                    } else {
                        v->s += t[p];
                    }
                    ++p;
                }
                if (p >= t.size()) fail("unterminated string");
                ++p;
            }
        } else {
            size_t s = p;
            while (p < t.size() && (isalnum((unsigned char)t[p]) || t[p] == '.' || t[p] == '-' || t[p] == '+')) ++p;
            std::string tok = t.substr(s, p - s);
            if (tok.empty()) fail(std::string("unexpected character '") + c + "'");
            std::string low;
            for (char ch : tok) low += (char)tolower((unsigned char)ch);
            if (low == "true" || low == "false") {
                v->type = Setting::Bool;
                v->b = low == "true";
            } else if (tok.find_first_of(".eE") != std::string::npos && low.rfind("0x", 0) != 0) {
                v->type = Setting::Float;
                v->f = strtod(tok.c_str(), nullptr);
            } else {
                v->type = Setting::Int;
                while (!tok.empty() && (tok.back() == 'L' || tok.back() == 'l')) tok.pop_back();
                char* end = nullptr;
                v->i = strtoll(tok.c_str(), &end, 0);
                if (!end || *end) fail("bad number '" + tok + "'");
            }
        }
        return v;
    }

    std::unique_ptr<Setting> setting()
    {
        std::string n = ident();
        skip();
        if (p < t.size() && (t[p] == '=' || t[p] == ':')) ++p;
        else fail("expected '=' or ':' after '" + n + "'");
        auto v = value();
        v->name = n;
        if (peek(';') || peek(',')) ++p;
        return v;
    }
};

}  // namespace

std::unique_ptr<Setting> parse_plan(const std::string& text)
{
    Parser ps(text);
    auto root = std::make_unique<Setting>();
    root->type = Setting::Group;
    for (;;) {
        ps.skip();
        if (ps.p >= text.size()) break;
        root->items.push_back(ps.setting());
    }
    return root;
}

std::unique_ptr<Setting> parse_plan_file(const std::string& path)
{
    std::ifstream in(path);
    if (!in) throw PlanError("cannot read plan file " + path);
    std::stringstream ss;
    ss << in.rdbuf();
    return parse_plan(ss.str());
}

}  // namespace pyg_host
