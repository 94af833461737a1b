// timefmt.h -- "[YYYY-mm-dd HH:MM:SS.mmm] " line prefix, the format of the
// reference's print_with_time (src/utils.cpp:14-30).
#pragma once

#include <stdarg.h>
#include <stdio.h>
#include <sys/time.h>
#include <time.h>

namespace nqb {

inline void print_with_time(const char *format, ...) {
    struct timeval tv;
    gettimeofday(&tv, nullptr);
    struct tm tmv;
    time_t secs = tv.tv_sec;
    localtime_r(&secs, &tmv);
    char buf[64];
    strftime(buf, sizeof(buf), "%Y-%m-%d %H:%M:%S", &tmv);
    printf("[%s.%03d] ", buf, (int)(tv.tv_usec / 1000));
    va_list ap;
    va_start(ap, format);
    vprintf(format, ap);
    va_end(ap);
}

inline double time_diff_ms(const struct timeval &a, const struct timeval &b) {
    return (b.tv_sec - a.tv_sec) * 1000.0 + (b.tv_usec - a.tv_usec) / 1000.0;
}

}  // namespace nqb
