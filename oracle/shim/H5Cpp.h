/* TEST INFRASTRUCTURE ONLY: empty stand-in for HDF5's C++ header (the oracle
 * build never writes HDF5). */
#ifndef ORC_SHIM_H5CPP_H
#define ORC_SHIM_H5CPP_H
#endif
