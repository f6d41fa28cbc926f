/*
 * TEST INFRASTRUCTURE ONLY.  Failure-returning definitions of the .apr file
 * helpers declared in the reference's io/hdf5functions_blosc.h, so that the
 * oracle build in oracle/_ref links without HDF5/blosc.  The oracle never
 * performs file IO; every helper reports failure.
 */
#include "io/hdf5functions_blosc.h"

void hdf5_register_blosc() {}
hid_t hdf5_create_file_blosc(std::string) { return -1; }
void hdf5_load_data_blosc(hid_t, void *, const char *) {}
void hdf5_load_data_blosc(hid_t, hid_t, void *, const char *) {}
void hdf5_write_attribute_blosc(hid_t, hid_t, const char *, hsize_t, hsize_t *, const void *const) {}
void hdf5_write_data_blosc(hid_t, hid_t, const char *, hsize_t, hsize_t *, void *, unsigned int, unsigned int, unsigned int) {}
void hdf5_write_data_standard(hid_t, hid_t, const char *, hsize_t, hsize_t *, void *) {}
void write_main_paraview_xdmf_xml(const std::string &, const std::string &, const std::string &, uint64_t) {}
void hdf5_load_data_blosc_partial(hid_t, void *, const char *, uint64_t, uint64_t) {}
void write_main_paraview_xdmf_xml_time(const std::string &, const std::string &, const std::string &, std::vector<uint64_t>) {}
void hdf5_write_data_blosc_create(hid_t, hid_t, const char *, hsize_t, hsize_t *, void *, unsigned int, unsigned int, unsigned int) {}
uint64_t hdf5_write_data_blosc_append(hid_t, hid_t, const char *, void *, hsize_t *) { return 0; }
void hdf5_write_data_blosc_partial(hid_t, void *, const char *, uint64_t, uint64_t) {}
void hdf5_create_dataset_blosc(hid_t, hid_t, const char *, hsize_t, hsize_t *, unsigned int, unsigned int, unsigned int) {}
bool attribute_exists(hid_t, const char *) { return false; }
bool group_exists(hid_t, const char *) { return false; }
bool data_exists(hid_t, const char *) { return false; }
