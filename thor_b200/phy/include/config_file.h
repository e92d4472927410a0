// Configuration keys of a physics module (the reference's config_file::append_config_var,
// src/headers/config_file.h:105-135): a key takes its default at registration; a value given later
// through thorx_phy_set_config (the .thr runner) is parsed into the registered variable.
#pragma once

#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <string>

class config_file
{
public:
    template<typename T> bool append_config_var(const std::string& name, T& target_, const T& default_val_) {
        if (setters.count(name))
            return false;
        target_       = default_val_;
        setters[name] = [&target_](const std::string& v) { return parse(v, target_); };
        return true;
    }
    // false when the key is unknown or the value does not parse
    bool set(const std::string& name, const std::string& value) {
        auto it = setters.find(name);
        return it != setters.end() && it->second(value);
    }

private:
    static bool parse(const std::string& v, bool& t) {
        if (v == "true" || v == "1") return t = true, true;
        if (v == "false" || v == "0") return t = false, true;
        return false;
    }
    static bool parse(const std::string& v, int& t) {
        char* e = nullptr;
        long  x = std::strtol(v.c_str(), &e, 10);
        return (e && *e == 0 && !v.empty()) ? (t = (int)x, true) : false;
    }
    static bool parse(const std::string& v, double& t) {
        char*  e = nullptr;
        double x = std::strtod(v.c_str(), &e);
        return (e && *e == 0 && !v.empty()) ? (t = x, true) : false;
    }
    static bool parse(const std::string& v, std::string& t) { return t = v, true; }
    std::map<std::string, std::function<bool(const std::string&)>> setters;
};
