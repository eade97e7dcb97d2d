// Fortran namelist input (the reference's input.nml: &FCInfo, &CrystalInfo, &AtmInfo, &AnhInfo,
// ... each closed by '/'), read the way a Fortran READ(nml=...) fills the variables it names:
//   name = values                 fills the variable from its first element in column-major order
//   name(i, j) = values           one element; name(:, j) = values a column (':' is the full
//                                 extent, 'a:b' a range); values fill the section in column order
// Values are separated by blanks or commas; r*v repeats v r times; strings are quoted with ' or ";
// logicals are .true./.false./T/F (with or without dots); '!' starts a comment.  Names are not
// case sensitive.  Variables the file does not name keep the caller's defaults.
#pragma once
#include <map>
#include <string>
#include <vector>

namespace nml {

struct Sub {
    int lo = 0, hi = 0;  // 1-based; full = true means ':'
    bool full = false;
};

struct Assign {
    std::vector<Sub> subs;
    std::vector<std::string> values;
};

struct Group {
    std::map<std::string, std::vector<Assign>> vars;  // lower-case name -> assignments in file order
    bool has(const std::string& name) const;
};

// Parse every group of a file.  Returns "" or an error message.
std::string parse_file(const std::string& path, std::map<std::string, Group>& out);
std::string parse_text(const std::string& text, std::map<std::string, Group>& out);

// Fill a Fortran array of shape dims (column-major) from the assignments of `name`; elements not
// assigned keep their values.  Returns "" or an error message.
std::string get(const Group& g, const std::string& name, const std::vector<int>& dims, std::vector<double>& a);
std::string get(const Group& g, const std::string& name, const std::vector<int>& dims, std::vector<int>& a);
std::string get(const Group& g, const std::string& name, const std::vector<int>& dims, std::vector<bool>& a);
std::string get(const Group& g, const std::string& name, const std::vector<int>& dims, std::vector<std::string>& a);
// Scalars.
std::string get(const Group& g, const std::string& name, double& v);
std::string get(const Group& g, const std::string& name, int& v);
std::string get(const Group& g, const std::string& name, bool& v);
std::string get(const Group& g, const std::string& name, std::string& v);

}  // namespace nml
