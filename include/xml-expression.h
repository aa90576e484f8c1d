/*
 * xml-expression.h -- XMLBIF 0.3 reader of the drop-in library.
 *
 * parse_xml_file replaces the reference's src/bnf-xml-parser/xml-expression.c:441-466
 * (declared in its xml-expression.h:8): same name, same argument, same
 * struct graph built in the same order, but read without libxml2, so a
 * reference driver (c_benchmark/main.c's XML path) links against libbp.so
 * alone.  The file must exist; a malformed document fails an assertion, as
 * the reference's reader does.
 */
#ifndef BP_XML_EXPRESSION_H_
#define BP_XML_EXPRESSION_H_

#include "graph.h"

#ifdef __cplusplus
extern "C" {
#endif

Graph_t parse_xml_file(const char *file_name);

#ifdef __cplusplus
}
#endif

#endif /* BP_XML_EXPRESSION_H_ */
