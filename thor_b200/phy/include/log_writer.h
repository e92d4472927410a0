// log::printf of the reference (src/headers/log_writer.h:100-150): module messages go to stdout.
#pragma once

#include <cstdio>

class log
{
public:
    template<typename... Args> static void printf(Args... args) {
#pragma GCC diagnostic push
#pragma GCC diagnostic ignored "-Wformat-security"
        std::printf(args...);
#pragma GCC diagnostic pop
    }
    template<typename... Args> static void printf_logonly(Args...) {}
    static void flush() { std::fflush(stdout); }
};
