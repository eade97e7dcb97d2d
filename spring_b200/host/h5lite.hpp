// h5lite: the subset of the HDF5 file format that SPRING's force-constant and output files use,
// written and read without the HDF5 library.
//
// The reference reads FC2nd_/FC3rd_/FC4th_<prefix><T>K_F.h5 (src/Kappa/Src/hdf5_wrap_mod.f90:40-337:
// datasets NumAtoms, atm_Indx and FC2 at the root; groups FC3rd / FC4th with one dataset
// FC3_mu<k> / FC4_mu<k> per basis atom) and writes kappa_<prefix><T>K.h5 (:650-766:
// ThermalConductivityTensor, LineWidth, PhaseSpace3rd, ...) through the Fortran HDF5 API, whose
// dataspaces list the Fortran dimensions in reverse and whose raw data is the Fortran array in
// memory order.  Those files use: a version 0 superblock, version 1 object headers, groups as
// symbol tables (a version 1 B-tree of symbol-table nodes plus a local heap), contiguous (or
// compact) data layout, and little-endian 32-bit integers or IEEE doubles.  This file implements
// exactly that (published format: "HDF5 File Format Specification Version 3.0"): the writer
// produces files the HDF5 library reads, the reader reads files of that shape written by the
// library (object-header continuation blocks included) and refuses anything else with a clear
// message.
#pragma once
#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace h5lite {

enum class Type { I32, F64 };

struct Dataset {
    Type type = Type::F64;
    std::vector<uint64_t> dims;  // HDF5 (C) order: the Fortran dimensions reversed
    std::vector<uint8_t> data;   // raw little-endian bytes, C order of dims (= Fortran memory order)
    size_t count() const {
        size_t n = 1;
        for (auto d : dims) n *= d;
        return n;
    }
};

struct Group {
    std::map<std::string, Dataset> datasets;
    std::map<std::string, std::unique_ptr<Group>> groups;
    Group& group(const std::string& name) {
        auto& g = groups[name];
        if (!g) g.reset(new Group());
        return *g;
    }
};

// Helpers for Fortran arrays: dims given in Fortran order (fastest first).
Dataset make_f64(const double* a, const std::vector<uint64_t>& fortran_dims);
Dataset make_i32(const int32_t* a, const std::vector<uint64_t>& fortran_dims);
std::vector<uint64_t> fortran_dims(const Dataset& d);

// Write `root` as a new file (truncating).  Returns "" or an error message.
std::string write_file(const std::string& path, const Group& root);
// Read a file into `root`.  Returns "" or an error message.
std::string read_file(const std::string& path, Group& root);

}  // namespace h5lite
