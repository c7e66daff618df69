/* Empty stand-in for libcurl's header. The reference's glob_funct.hpp
 * includes <curl/curl.h> for licence-check helpers that the cell models
 * never call; this stub lets the model sources compile without libcurl. */
#ifndef CEP_ORACLE_CURL_STUB_H
#define CEP_ORACLE_CURL_STUB_H
typedef int CURLcode;
typedef void CURL;
#endif
