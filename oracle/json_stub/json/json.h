/*
 * Test infrastructure only: minimal stand-in for JsonCpp's <json/json.h>.
 * The G2S reference sources compiled for the CPU oracle only need the type
 * name Json::Value (a typedef in G2S include/jobManager.hpp:40); nothing is
 * parsed or serialised, because the distributed/server code paths that use
 * JSON are compiled out.
 */
#ifndef G2S_B200_JSON_STUB_H
#define G2S_B200_JSON_STUB_H
namespace Json {
class Value {};
}
#endif
