// Link stubs for the reference's HDF5 reader classes (EMhdf, EMhdf2; declared in
// include/EMReader/emhdf.h and emhdf2.h), so that the reference's emdata.cpp compiles and
// links without libhdf5 for the projection harness (TEST INFRASTRUCTURE ONLY; libhdf5 is not
// in this image).  MRC inputs never reach them: is_valid says "not HDF" and every other
// member aborts if ever called.
#include <cstdio>
#include <cstdlib>

#include "emhdf.h"
#include "emhdf2.h"

namespace {
[[noreturn]] void unreachable(const char* what) {
  std::fprintf(stderr, "HDF5 reader stub %s called: this harness reads MRC files only\n", what);
  std::abort();
}
}  // namespace

EMhdf::EMhdf(const char*, const char*) { unreachable("EMhdf::EMhdf"); }
EMhdf::~EMhdf() {}
int EMhdf::init_test(const char*) { unreachable("EMhdf::init_test"); }
int EMhdf::is_valid(const char*) { return 0; }
int* EMhdf::read_dims(int, int*) { unreachable("EMhdf::read_dims"); }
int EMhdf::read_data(int, float**) { unreachable("EMhdf::read_data"); }
int EMhdf::read_int_attr(int, const char*) { unreachable("EMhdf::read_int_attr"); }
float EMhdf::read_float_attr(int, const char*) { unreachable("EMhdf::read_float_attr"); }
const char* EMhdf::read_string_attr(int, const char*) { unreachable("EMhdf::read_string_attr"); }
void EMhdf::read_array_attr(int, const char*, void*) { unreachable("EMhdf::read_array_attr"); }
int EMhdf::read_euler_attr(int, const char*) { unreachable("EMhdf::read_euler_attr"); }
int EMhdf::read_ctfit(int, CTFParam*) { unreachable("EMhdf::read_ctfit"); }
int EMhdf::read_mapinfo_attr(int, const char*) { unreachable("EMhdf::read_mapinfo_attr"); }

EMhdf2::EMhdf2(const char*, const char*) { unreachable("EMhdf2::EMhdf2"); }
EMhdf2::~EMhdf2() {}
emdataHeader* EMhdf2::read_header(int, Euler&) { unreachable("EMhdf2::read_header"); }
int EMhdf2::read_data(float*, int) { unreachable("EMhdf2::read_data"); }
int EMhdf2::write_header(const emdataHeader&, int, const Euler&) { unreachable("EMhdf2::write_header"); }
int EMhdf2::write_data(const float* const, int) { unreachable("EMhdf2::write_data"); }
int EMhdf2::get_num_dataset() { unreachable("EMhdf2::get_num_dataset"); }
