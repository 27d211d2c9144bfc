// ref_io_stubs.cu -- stand-ins for the reference's HDF5 snapshot I/O
// (src/io/hdf5_io.cu) and the shearing-box unshear output
// (src/io/unshear_output.cu), which need libhdf5 / HighFive, absent here.
// The timing driver (ref_driver.cu) never writes or reads a snapshot; these
// definitions only let the reference's other sources link, and fail loudly
// if anything does call them.
#include <cstdio>
#include <cstdlib>
#include <string>

#include "common.hpp"
#include "inputoutput.hpp"

void InputOutput::WriteDataFile() {
    std::fprintf(stderr, "reference timing build: snapshot output is not built (no HDF5 library)\n");
    std::exit(3);
}

void InputOutput::ReadDataFile(int) {
    std::fprintf(stderr, "reference timing build: restart input is not built (no HDF5 library)\n");
    std::exit(3);
}

void InputOutput::UnshearOutput(data_type*, scalar_type*, double) {
    std::fprintf(stderr, "reference timing build: the shearing-box output is not built\n");
    std::exit(3);
}

void InputOutput::UnshearField(data_type*, double) {
    std::fprintf(stderr, "reference timing build: the shearing-box output is not built\n");
    std::exit(3);
}

int fileCounter(std::string) { return 0; }
