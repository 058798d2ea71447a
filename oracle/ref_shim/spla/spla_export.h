/* Symbol visibility for the oracle build of the reference host library
 * (normally generated by CMake's GenerateExportHeader). Test infrastructure. */
#ifndef SPLA_EXPORT_H
#define SPLA_EXPORT_H
#define SPLA_EXPORT __attribute__((visibility("default")))
#endif
