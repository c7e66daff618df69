/* TEST INFRASTRUCTURE ONLY: CEPCell_NEO/modules/commons.cpp includes
 * libmagic's header but calls none of its functions. */
#ifndef CEP_STUB_MAGIC_H
#define CEP_STUB_MAGIC_H
#endif
