// CPU ORACLE — test infrastructure. Empty stand-in: the reference headers
// compiled by the oracle include rapidjson but use none of its names.
#pragma once
