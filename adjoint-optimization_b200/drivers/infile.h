// infile.h -- reader of the reference's driver configuration files.
//
// The reference's drivers read `infile_grad` / `infile_forward`: MATLAB
// assignment lines `name = value; % comment`, evaluated one by one for the
// names a driver asks for; other lines are reported as "not evaluated", and a
// missing name is an error that lists every missing one
// (src/cuda/read_check_2.m:1-50, called from simple_grad_desc.m:30-35 and
// save_fk_forward_Et.m:36-41).  This reader accepts the value forms those
// files use: numbers, row vectors `[a, b, c]`, quoted strings (with '' for a
// quote) and function handles `@name` (kept as the name).
#pragma once

#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace fkadj_drivers {

struct Value {
    enum Kind { NUM, VEC, STR, HANDLE } kind = NUM;
    std::vector<double> nums;  // NUM: one value; VEC: all
    std::string str;           // STR and HANDLE
};

class Infile {
   public:
    // Parses the file; unknown lines are printed (as the reference does) only
    // when they do not assign one of `wanted` or `optional`.
    Infile(const std::string& path, const std::vector<std::string>& wanted,
           const std::vector<std::string>& optional = {}) {
        FILE* f = fopen(path.c_str(), "r");
        if (!f) throw std::runtime_error("cannot open configuration file '" + path + "'");
        std::string line;
        int c;
        while (true) {
            line.clear();
            while ((c = fgetc(f)) != EOF && c != '\n') line.push_back((char)c);
            handle(line, wanted, optional);
            if (c == EOF) break;
        }
        fclose(f);
        std::string missing;
        for (const auto& w : wanted)
            if (!vals_.count(w)) missing += w + " ";
        if (!missing.empty())
            throw std::runtime_error("The following variables were not found: " + missing);
    }

    bool has(const std::string& k) const { return vals_.count(k) != 0; }
    const Value& get(const std::string& k) const {
        auto it = vals_.find(k);
        if (it == vals_.end()) throw std::runtime_error("variable '" + k + "' not set");
        return it->second;
    }
    double num(const std::string& k) const {
        const Value& v = get(k);
        if (v.kind != Value::NUM) throw std::runtime_error("'" + k + "' must be a number");
        return v.nums[0];
    }
    double num_or(const std::string& k, double d) const { return has(k) ? num(k) : d; }
    std::vector<double> vec(const std::string& k) const {
        const Value& v = get(k);
        if (v.kind != Value::VEC && v.kind != Value::NUM)
            throw std::runtime_error("'" + k + "' must be numeric");
        return v.nums;
    }
    std::string str(const std::string& k) const {
        const Value& v = get(k);
        if (v.kind != Value::STR && v.kind != Value::HANDLE)
            throw std::runtime_error("'" + k + "' must be a string");
        return v.str;
    }
    std::string str_or(const std::string& k, const std::string& d) const {
        return has(k) ? str(k) : d;
    }

   private:
    std::map<std::string, Value> vals_;

    static std::string trim(const std::string& s) {
        size_t a = 0, b = s.size();
        while (a < b && isspace((unsigned char)s[a])) ++a;
        while (b > a && isspace((unsigned char)s[b - 1])) --b;
        return s.substr(a, b - a);
    }

    // Drops a '%' comment that is not inside a quoted string.
    static std::string strip_comment(const std::string& s) {
        bool q = false;
        for (size_t i = 0; i < s.size(); ++i) {
            if (s[i] == '\'') q = !q;
            else if (s[i] == '%' && !q) return s.substr(0, i);
        }
        return s;
    }

    static bool parse_value(std::string t, Value& v) {
        t = trim(t);
        while (!t.empty() && t.back() == ';') t = trim(t.substr(0, t.size() - 1));
        if (t.empty()) return false;
        if (t[0] == '\'') {
            v.kind = Value::STR;
            for (size_t i = 1; i < t.size(); ++i) {
                if (t[i] == '\'') {
                    if (i + 1 < t.size() && t[i + 1] == '\'') {
                        v.str.push_back('\'');
                        ++i;
                        continue;
                    }
                    return trim(t.substr(i + 1)).empty();
                }
                v.str.push_back(t[i]);
            }
            return false;  // unterminated
        }
        if (t[0] == '@') {
            v.kind = Value::HANDLE;
            v.str = trim(t.substr(1));
            return !v.str.empty();
        }
        std::string body = t;
        if (t[0] == '[') {
            if (t.back() != ']') return false;
            v.kind = Value::VEC;
            body = t.substr(1, t.size() - 2);
        }
        for (char& ch : body)
            if (ch == ',') ch = ' ';
        const char* p = body.c_str();
        while (true) {
            while (*p && isspace((unsigned char)*p)) ++p;
            if (!*p) break;
            char* end;
            const double x = strtod(p, &end);
            if (end == p) return false;
            v.nums.push_back(x);
            p = end;
        }
        if (v.kind == Value::NUM && v.nums.size() != 1) return false;
        return !v.nums.empty() || v.kind == Value::VEC;
    }

    void handle(const std::string& raw, const std::vector<std::string>& wanted,
                const std::vector<std::string>& optional) {
        const std::string line = trim(strip_comment(raw));
        if (line.empty()) return;
        size_t k = 0;
        while (k < line.size() && (isalnum((unsigned char)line[k]) || line[k] == '_')) ++k;
        const std::string name = line.substr(0, k);
        size_t e = k;
        while (e < line.size() && line[e] == ' ') ++e;
        bool known = false;
        for (const auto& w : wanted) known |= (w == name);
        for (const auto& w : optional) known |= (w == name);
        if (name.empty() || e >= line.size() || line[e] != '=' || !known || vals_.count(name)) {
            printf("Expression '%s' not evaluated\n", raw.c_str());
            return;
        }
        Value v;
        if (!parse_value(line.substr(e + 1), v))
            throw std::runtime_error("cannot evaluate '" + raw + "'");
        vals_[name] = v;
    }
};

// float_integer (src/cuda/float_integer.m:1-13): r must be an integer to
// within 5e-16 relative.
inline long long float_integer(double r) {
    if (r == 0) return 0;
    const double rn = std::round(r);
    if (std::fabs(r - rn) < 5e-16 * r) return (long long)rn;
    throw std::runtime_error("Not a float integer");
}

}  // namespace fkadj_drivers
