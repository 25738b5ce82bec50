/* Compile-only stand-in: DiffOper.cxx includes this header but uses none of its ITK-based I/O. */
#include "AtlasWerksTypes.h"
