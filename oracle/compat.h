/* Force-included into every translation unit of the reference serial build
 * made by oracle/Makefile (test infrastructure only; nothing in the product
 * links it).
 *
 * The reference pins fmt 8.0.1 / spdlog 1.9.2 (ARTSS compile.sh:199-212).
 * The only spdlog available offline is 1.14.1 with bundled fmt 10.2.1, and
 * fmt >= 10 refuses to format unscoped enums implicitly.  These overloads
 * give fmt an explicit integer view of the five enums the reference logs
 * (src/utility/Mapping.h:16-63); they change no arithmetic. */
#ifndef ARTSS_ORACLE_COMPAT_H
#define ARTSS_ORACLE_COMPAT_H
#ifdef __cplusplus
#include "src/utility/Mapping.h"
inline int format_as(Patch v) { return static_cast<int>(v); }
inline int format_as(BoundaryCondition v) { return static_cast<int>(v); }
inline int format_as(FieldType v) { return static_cast<int>(v); }
inline int format_as(CoordinateAxis v) { return static_cast<int>(v); }
inline int format_as(State v) { return static_cast<int>(v); }
#endif
#endif
