// Stand-in for BOINC's MFILE (buffered output file): here a plain stdio
// stream, flushed on flush() and close().  Test infrastructure only.
#pragma once
#include <cstdio>

class MFILE {
    FILE* f_ = nullptr;

public:
    int open(const char* path, const char* mode);
    int printf(const char* format, ...) __attribute__((format(printf, 2, 3)));
    int flush(void);
    int close(void);
};
