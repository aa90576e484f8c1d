/*
 * ref_bif.c -- TEST INFRASTRUCTURE ONLY.  Loads a BIF network with the
 * reference's own vendored bison/flex parser (src/bnf-parser/Parser.c,
 * Lexer.c, expression.c; entry sequence as in c_benchmark/main.c:166-182)
 * and returns the Graph_t that build_graph (expression.c:919-937) makes.
 *
 * The same object links either against the reference's graph.c (the
 * checker) or against this project's libbp.so (the drop-in check: the
 * reference parser, compiled against the reference header, building a graph
 * inside the CUDA-backed library).
 */
#include <stdio.h>
#include <stdlib.h>

#include "expression.h"
#include "Parser.h"
#include "Lexer.h"

int yyparse(struct expression **expr, yyscan_t scanner);

Graph_t refbif_load(const char *path)
{
    struct expression *expression = NULL;
    yyscan_t scanner;
    FILE *in = fopen(path, "r");
    if (!in)
        return NULL;
    if (yylex_init(&scanner) != 0) {
        fclose(in);
        return NULL;
    }
    yyset_in(in, scanner);
    int rc = yyparse(&expression, scanner);
    yylex_destroy(scanner);
    fclose(in);
    if (rc != 0 || expression == NULL)
        return NULL;
    Graph_t g = build_graph(expression);
    delete_expression(expression);
    return g;
}
