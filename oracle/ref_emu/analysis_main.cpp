// analysis_main.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Runs the reference's own analysis code (src/sphere.cpp: DEM::porosity,
// DEM::printContacts -> DEM::findOverlaps) on a .bin file, with the DEM
// object constructed as src/porosity.cpp:72 does (no CUDA set-up, no
// fluid), and prints with 17 significant digits so that the output pins
// the FP64 values.
//   sphere_analysis_ref porosity <file.bin> <slices>
//   sphere_analysis_ref contacts <file.bin>
#include <cstdlib>
#include <iostream>
#include <string>

#include "sphere.h"

int main(int argc, char **argv)
{
    if (argc < 3) {
        std::cerr << "usage: " << argv[0] << " porosity|contacts <file.bin> [slices]\n";
        return 2;
    }
    std::cout.precision(17);
    DEM dem(argv[2], 0, 0, 0, 0, 0);
    const std::string what = argv[1];
    if (what == "porosity") dem.porosity(argc > 3 ? std::atoi(argv[3]) : 10);
    else if (what == "contacts") dem.printContacts();
    else return 2;
    return 0;
}
