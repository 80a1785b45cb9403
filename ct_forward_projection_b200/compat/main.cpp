// main.cpp — command-line entry, the reference's
// Source/Main_Forward_Projection_V1.1.cpp:18-39: runs the projector selected
// by Config/ScanSetting.ini in the working directory (or the directory given
// as the first argument).  A configuration or input error prints a message and
// exits with status 1.
#include <exception>
#include <iostream>

#include "ForwardProjection.h"

int main(int argc, char** argv)
{
    try {
        ForwardProjection fp;
        if (argc > 1) fp.baseDir = argv[1];
        fp.run();
    } catch (const std::exception& e) {
        std::cerr << "error: " << e.what() << std::endl;
        return 1;
    }
    return 0;
}
