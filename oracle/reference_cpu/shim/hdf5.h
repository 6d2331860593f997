/* TEST INFRASTRUCTURE ONLY.
 *
 * The one HDF5 type that the reference's module headers name.  The harness
 * does not write HDF5 files: the mesh module's output routine is linked
 * against no-op stand-ins (ref_driver.cc). */
#pragma once

typedef long long hid_t;
