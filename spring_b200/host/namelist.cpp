// Fortran namelist reader: see namelist.hpp.
#include "namelist.hpp"

#include <algorithm>
#include <cctype>
#include <cstdlib>
#include <fstream>
#include <sstream>

namespace nml {
namespace {

std::string lower(std::string s) {
    for (auto& c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

// Tokens of a value list: quoted strings stay whole (quotes removed, '' -> '), r*v expands.
std::string split_values(const std::string& s, std::vector<std::string>& out) {
    size_t i = 0;
    while (i < s.size()) {
        const char c = s[i];
        if (std::isspace((unsigned char)c) || c == ',') {
            ++i;
            continue;
        }
        std::string tok;
        if (c == '\'' || c == '"') {
            const char q = c;
            ++i;
            for (;;) {
                if (i >= s.size()) return "unterminated string";
                if (s[i] == q) {
                    if (i + 1 < s.size() && s[i + 1] == q) {
                        tok.push_back(q);
                        i += 2;
                        continue;
                    }
                    ++i;
                    break;
                }
                tok.push_back(s[i++]);
            }
            out.push_back("\x01" + tok);  // marks a quoted string
            continue;
        }
        while (i < s.size() && !std::isspace((unsigned char)s[i]) && s[i] != ',') tok.push_back(s[i++]);
        const size_t star = tok.find('*');
        if (star != std::string::npos && star > 0 &&
            std::all_of(tok.begin(), tok.begin() + star, [](char ch) { return std::isdigit((unsigned char)ch); })) {
            const int r = std::atoi(tok.substr(0, star).c_str());
            std::string v = tok.substr(star + 1);
            if (!v.empty() && (v[0] == '\'' || v[0] == '"') && v.size() >= 2) v = "\x01" + v.substr(1, v.size() - 2);
            for (int k = 0; k < r; ++k) out.push_back(v);
            continue;
        }
        out.push_back(tok);
    }
    return "";
}

std::string parse_subs(const std::string& s, std::vector<Sub>& subs) {
    std::stringstream ss(s);
    std::string part;
    while (std::getline(ss, part, ',')) {
        part.erase(std::remove_if(part.begin(), part.end(), [](char ch) { return std::isspace((unsigned char)ch); }),
                   part.end());
        Sub u;
        if (part == ":") {
            u.full = true;
        } else {
            const size_t colon = part.find(':');
            if (colon == std::string::npos) {
                u.lo = u.hi = std::atoi(part.c_str());
            } else {
                u.lo = std::atoi(part.substr(0, colon).c_str());
                u.hi = std::atoi(part.substr(colon + 1).c_str());
            }
            if (u.lo < 1 || u.hi < u.lo) return "bad subscript '" + part + "'";
        }
        subs.push_back(u);
    }
    return "";
}

bool to_bool(const std::string& t, bool& v) {
    std::string s = lower(t);
    if (!s.empty() && s[0] == '.') s = s.substr(1);
    if (s.empty()) return false;
    if (s[0] == 't') { v = true; return true; }
    if (s[0] == 'f') { v = false; return true; }
    return false;
}

bool to_double(const std::string& t, double& v) {
    if (t.empty() || t[0] == '\x01') return false;
    std::string s = t;
    for (auto& c : s)
        if (c == 'd' || c == 'D') c = 'e';  // Fortran double-precision exponent
    char* end = nullptr;
    v = std::strtod(s.c_str(), &end);
    return end && *end == 0;
}

template <class T, class Conv>
std::string fill(const Group& g, const std::string& name, const std::vector<int>& dims, std::vector<T>& a, Conv conv) {
    size_t total = 1;
    for (int d : dims) total *= (size_t)d;
    if (a.size() < total) a.resize(total);
    auto it = g.vars.find(lower(name));
    if (it == g.vars.end()) return "";
    for (const Assign& as : it->second) {
        // the element offsets of the section, in column-major order
        std::vector<size_t> offs;
        if (as.subs.empty()) {
            for (size_t k = 0; k < total; ++k) offs.push_back(k);
        } else {
            if (as.subs.size() != dims.size()) return name + ": wrong number of subscripts";
            std::vector<int> lo(dims.size()), hi(dims.size());
            for (size_t d = 0; d < dims.size(); ++d) {
                lo[d] = as.subs[d].full ? 1 : as.subs[d].lo;
                hi[d] = as.subs[d].full ? dims[d] : as.subs[d].hi;
                if (hi[d] > dims[d]) return name + ": subscript out of range";
            }
            std::vector<int> idx(lo);
            for (;;) {
                size_t off = 0, stride = 1;
                for (size_t d = 0; d < dims.size(); ++d) {
                    off += (size_t)(idx[d] - 1) * stride;
                    stride *= (size_t)dims[d];
                }
                offs.push_back(off);
                size_t d = 0;
                while (d < dims.size() && ++idx[d] > hi[d]) {
                    idx[d] = lo[d];
                    ++d;
                }
                if (d == dims.size()) break;
            }
        }
        if (as.values.size() > offs.size()) return name + ": more values than elements";
        for (size_t k = 0; k < as.values.size(); ++k) {
            T v;
            if (!conv(as.values[k], v)) return name + ": cannot read value '" + as.values[k] + "'";
            a[offs[k]] = v;
        }
    }
    return "";
}

}  // namespace

bool Group::has(const std::string& name) const { return vars.count(lower(name)) > 0; }

std::string parse_text(const std::string& text, std::map<std::string, Group>& out) {
    // strip comments (outside strings) and join the lines
    std::string s;
    {
        char q = 0;
        for (size_t i = 0; i < text.size(); ++i) {
            const char c = text[i];
            if (q) {
                if (c == q) q = 0;
                s.push_back(c);
            } else if (c == '\'' || c == '"') {
                q = c;
                s.push_back(c);
            } else if (c == '!') {
                while (i < text.size() && text[i] != '\n') ++i;
                s.push_back('\n');
            } else {
                s.push_back(c);
            }
        }
    }
    size_t i = 0;
    while ((i = s.find('&', i)) != std::string::npos) {
        size_t j = i + 1;
        while (j < s.size() && (std::isalnum((unsigned char)s[j]) || s[j] == '_')) ++j;
        const std::string gname = lower(s.substr(i + 1, j - i - 1));
        // the group body ends at the first '/' outside a string
        size_t k = j;
        char q = 0;
        for (; k < s.size(); ++k) {
            if (q) {
                if (s[k] == q) q = 0;
            } else if (s[k] == '\'' || s[k] == '"') {
                q = s[k];
            } else if (s[k] == '/') {
                break;
            }
        }
        if (k >= s.size()) return "namelist group &" + gname + " is not closed by '/'";
        const std::string body = s.substr(j, k - j);
        Group& g = out[gname];
        // split the body at each "name [(subs)] =" that starts an assignment
        std::vector<std::pair<size_t, size_t>> heads;  // (start of name, position of '=')
        q = 0;
        for (size_t p = 0; p < body.size(); ++p) {
            if (q) {
                if (body[p] == q) q = 0;
                continue;
            }
            if (body[p] == '\'' || body[p] == '"') {
                q = body[p];
                continue;
            }
            if (body[p] != '=') continue;
            size_t e = p;  // walk back over "(subs)" and the name
            while (e > 0 && std::isspace((unsigned char)body[e - 1])) --e;
            if (e > 0 && body[e - 1] == ')') {
                int depth = 0;
                while (e > 0) {
                    --e;
                    if (body[e] == ')') ++depth;
                    if (body[e] == '(' && --depth == 0) break;
                }
                while (e > 0 && std::isspace((unsigned char)body[e - 1])) --e;
            }
            size_t b = e;
            while (b > 0 && (std::isalnum((unsigned char)body[b - 1]) || body[b - 1] == '_' || body[b - 1] == '%')) --b;
            if (b == e) return "&" + gname + ": '=' without a variable name";
            heads.push_back({b, p});
        }
        for (size_t h = 0; h < heads.size(); ++h) {
            const size_t b = heads[h].first, eq = heads[h].second;
            const size_t vend = h + 1 < heads.size() ? heads[h + 1].first : body.size();
            std::string lhs = body.substr(b, eq - b);
            Assign as;
            const size_t par = lhs.find('(');
            std::string name = lhs.substr(0, par);
            name.erase(std::remove_if(name.begin(), name.end(), [](char ch) { return std::isspace((unsigned char)ch); }),
                       name.end());
            if (par != std::string::npos) {
                const size_t cl = lhs.rfind(')');
                const std::string e = parse_subs(lhs.substr(par + 1, cl - par - 1), as.subs);
                if (!e.empty()) return "&" + gname + " " + name + ": " + e;
            }
            const std::string e = split_values(body.substr(eq + 1, vend - eq - 1), as.values);
            if (!e.empty()) return "&" + gname + " " + name + ": " + e;
            g.vars[lower(name)].push_back(as);
        }
        i = k + 1;
    }
    return "";
}

std::string parse_file(const std::string& path, std::map<std::string, Group>& out) {
    std::ifstream in(path);
    if (!in) return "cannot open namelist file " + path;
    std::stringstream ss;
    ss << in.rdbuf();
    return parse_text(ss.str(), out);
}

std::string get(const Group& g, const std::string& name, const std::vector<int>& dims, std::vector<double>& a) {
    return fill(g, name, dims, a, [](const std::string& t, double& v) { return to_double(t, v); });
}
std::string get(const Group& g, const std::string& name, const std::vector<int>& dims, std::vector<int>& a) {
    return fill(g, name, dims, a, [](const std::string& t, int& v) {
        double d;
        if (!to_double(t, d) || d != (double)(long long)d) return false;
        v = (int)d;
        return true;
    });
}
std::string get(const Group& g, const std::string& name, const std::vector<int>& dims, std::vector<bool>& a) {
    std::vector<char> tmp(a.begin(), a.end());
    std::string e = fill(g, name, dims, tmp, [](const std::string& t, char& v) {
        bool b;
        if (!to_bool(t[0] == '\x01' ? t.substr(1) : t, b)) return false;
        v = b;
        return true;
    });
    a.assign(tmp.begin(), tmp.end());
    return e;
}
std::string get(const Group& g, const std::string& name, const std::vector<int>& dims, std::vector<std::string>& a) {
    return fill(g, name, dims, a, [](const std::string& t, std::string& v) {
        v = t[0] == '\x01' ? t.substr(1) : t;
        return true;
    });
}
std::string get(const Group& g, const std::string& name, double& v) {
    std::vector<double> a{v};
    std::string e = get(g, name, {1}, a);
    v = a[0];
    return e;
}
std::string get(const Group& g, const std::string& name, int& v) {
    std::vector<int> a{v};
    std::string e = get(g, name, {1}, a);
    v = a[0];
    return e;
}
std::string get(const Group& g, const std::string& name, bool& v) {
    std::vector<bool> a{v};
    std::string e = get(g, name, {1}, a);
    v = a[0];
    return e;
}
std::string get(const Group& g, const std::string& name, std::string& v) {
    std::vector<std::string> a{v};
    std::string e = get(g, name, {1}, a);
    v = a[0];
    return e;
}

}  // namespace nml
