// Forced-include shim that lets the reference's Windows/MSVC host sources
// compile on Linux for the reference build (oracle/build_ref.sh).  TEST
// INFRASTRUCTURE ONLY.  It maps the MSVC CRT calls the reference uses to POSIX
// ones and reproduces the MSVC rand()/srand() generator, which the reference
// relies on for its seeded scintillator thickness (CBCTForwardProj.cpp:101).
#pragma once
#include <cmath>
#include <math.h>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sys/stat.h>
#include <sys/types.h>
#include <unistd.h>

#define sprintf_s(buf, size, ...) snprintf((buf), (size), __VA_ARGS__)
#define _access(path, mode) access((path), (mode))
#define _mkdir(path) mkdir((path), 0755)

// "pause" waits for a key press on Windows; here it is a no-op.
static inline int ctfp_ref_system(const char*) { return 0; }
#define system(cmd) ctfp_ref_system(cmd)

// MSVC CRT generator: state = state * 214013 + 2531011, output (state >> 16) & 0x7fff.
static unsigned int ctfp_ref_rand_state = 1u;
static inline void ctfp_ref_srand(unsigned int seed) { ctfp_ref_rand_state = seed; }
static inline int ctfp_ref_rand(void)
{
    ctfp_ref_rand_state = ctfp_ref_rand_state * 214013u + 2531011u;
    return (int)((ctfp_ref_rand_state >> 16) & 0x7fffu);
}
#define srand(s) ctfp_ref_srand(s)
#define rand() ctfp_ref_rand()
