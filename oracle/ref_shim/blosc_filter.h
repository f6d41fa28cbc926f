/* TEST INFRASTRUCTURE ONLY: empty stand-in for the blosc HDF5 filter header (blosc is not installed). */
