// HDF5 files of the reference's output and restart layout, without libhdf5: the shape the
// reference's storage class writes (src/headers/storage.h:54-230, H5Cpp with default properties):
// one flat root group of 1-D datasets, IEEE F64LE or STD_I32LE, each with the two scalar
// fixed-length string attributes "Variable" (the description) and "units".
//
// The writer produces the byte layout of thor_b200/h5.py (the same superblock v0, root symbol
// table, B-tree, local heap, symbol-table nodes, object headers v1 and contiguous data, at the
// same addresses), so files from either runner differ only in their modification-time messages.
// The reader takes what the library writes for these files: v0 superblocks, symbol-table groups
// (B-trees of any depth), object headers v1 with continuation messages, dataspace v1/v2,
// fixed-point, floating-point and string datatypes, contiguous and compact layouts, attribute
// messages v1-v3 (The HDF Group, "HDF5 File Format Specification").
#pragma once

#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace thorx_h5 {

struct Dataset {
    bool                               integer = false; // stored as a fixed-point type
    std::vector<double>                values;          // every element, converted to double
    std::vector<uint64_t>              shape;           // empty: scalar
    std::map<std::string, std::string> attrs;           // string attributes (Variable, units)
};

class Writer {
  public:
    // A 1-D dataset of doubles (F64LE) or of 32-bit integers (STD_I32LE).
    void table(const std::string& name, const double* v, size_t n, const std::string& unit,
               const std::string& description);
    void table_i32(const std::string& name, const int32_t* v, size_t n, const std::string& unit,
                   const std::string& description);
    void value(const std::string& name, double v, const std::string& unit,
               const std::string& description);
    void value_i32(const std::string& name, int32_t v, const std::string& unit,
                   const std::string& description);
    // Writes the file (path + ".tmp", then renamed over path). False with *err on failure.
    bool close(const std::string& path, std::string* err);

  private:
    struct Item {
        bool                 integer;
        std::vector<uint8_t> raw; // little-endian element bytes
        std::string          unit, description;
    };
    std::map<std::string, Item> items_; // names without the leading '/', in strcmp order
};

// Every dataset of the root group by name. False with *err if the file is not one this reader
// takes.
bool read(const std::string& path, std::map<std::string, Dataset>& out, std::string* err);

} // namespace thorx_h5
