// gvaconvert <graph>.g <out prefix>: writes <prefix>.mygraph, <prefix>.metadata
// and <prefix>.reorder exactly as the reference converter (tools/genDatabase.cpp)
// does for the same .g file.
#include <cstdio>
#include <string>

#include "../../include/geneva.h"

int main(int argc, char** argv) {
    if (argc != 3) {
        std::printf("usage: %s <graph>.g <out prefix>\n", argv[0]);
        return 1;
    }
    const std::string p = argv[2];
    int st = gva_convert_g(argv[1], (p + ".mygraph").c_str(), (p + ".metadata").c_str(), (p + ".reorder").c_str());
    if (st) {
        std::printf("error: %s\n", gva_last_error());
        return 1;
    }
    return 0;
}
