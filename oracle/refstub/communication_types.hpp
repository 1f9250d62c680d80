// Test infrastructure only (oracle build). linpack_data.cpp includes this
// header but uses none of its names; an empty stand-in keeps the include of
// shared/include/communication_types.hpp out of the oracle build.
#ifndef ORACLE_REFSTUB_COMMUNICATION_TYPES_HPP
#define ORACLE_REFSTUB_COMMUNICATION_TYPES_HPP
#endif
