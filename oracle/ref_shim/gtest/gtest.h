/* Empty stand-in: the PittPack tree includes gtest but defines no tests.
 * TEST INFRASTRUCTURE ONLY (oracle/_ref). */
#ifndef PP_SHIM_GTEST_H
#define PP_SHIM_GTEST_H
#endif
