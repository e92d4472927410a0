// The HDF5 output wrapper a module's store hooks write to (the reference's storage,
// src/headers/storage.h:54-230). thorx writes its output files from the runner
// (thor_b200/esp.py, thor_b200/h5.py); module tables handed to this class are not written, and a
// module's restart read (init_data with a storage) finds no table.
#pragma once

#include <memory>
#include <string>

class storage
{
public:
    storage(const std::string& = "", const bool& = false) {}
    bool has_table(const std::string&) { return false; }
    template<typename T>
    void append_table(T*, const int&, std::string, std::string, std::string) {}
    template<typename T> void append_value(T, std::string, std::string, std::string) {}
    template<typename T> bool read_table(const std::string&, std::unique_ptr<T[]>&, int&) { return false; }
    template<typename T> bool read_table_to_ptr(const std::string&, T*, int) { return false; }
    bool is_open() { return false; }
};
