/*
 * xmlbif.c -- parse_xml_file: XMLBIF 0.3 networks into a struct graph,
 * without libxml2.
 *
 * Replaces the reference's src/bnf-xml-parser/xml-expression.c:441-466,
 * which reads the document with libxml2 and XPath.  This file tokenises the
 * XML itself (elements, attributes skipped, text, comments, CDATA, the
 * predefined and numeric character references, a DOCTYPE with an internal
 * subset) into a small element tree, then builds the graph through this
 * library's own graph.h calls in the reference's order:
 *
 *   create_graph(#VARIABLE, 2 * #GIVEN)                         (:453-456)
 *   per VARIABLE, in document order: the text of every OUTCOME text node
 *     into variable_names, then graph_add_node(#outcomes, NAME)  (:142-211)
 *   per DEFINITION without GIVEN: the numbers of the TABLE's last text
 *     node (sscanf "%f") to graph_set_node_state                (:283-318)
 *   per DEFINITION with GIVENs: the CPT marginalised onto each parent from
 *     the last GIVEN to the first, with the reference's strided float sums,
 *     then graph_add_edge parent -> child and, unless the parent is
 *     observed, child -> parent with the transposed table     (:331-419)
 *
 * Text is taken as libxml2 hands it over (no trimming): a name's text node
 * is compared byte for byte by find_node_by_name.  The reference reads CPT
 * entries past the end of the table in its strided sum (undefined); here
 * they count as 0, as in the test restatement.
 */
#include <assert.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "constants.h"
#include "graph.h"
#include "xml-expression.h"

typedef struct xnode {
    char *tag;                 /* element name */
    struct xnode **kids;       /* child elements, document order */
    unsigned nkids, capkids;
    char **texts;              /* text node children, document order */
    unsigned ntexts, captexts;
} xnode;

typedef struct {
    const char *s;
    size_t n, i;
    int bad;
} xscan;

static void *xgrow(void *p, unsigned *cap, size_t elem) {
    unsigned c = *cap ? 2 * *cap : 8;
    void *q = realloc(p, (size_t)c * elem);
    if (!q) {
        fprintf(stderr, "parse_xml_file: out of memory\n");
        abort();
    }
    *cap = c;
    return q;
}

static void xadd_kid(xnode *p, xnode *k) {
    if (p->nkids == p->capkids) p->kids = (xnode **)xgrow(p->kids, &p->capkids, sizeof(xnode *));
    p->kids[p->nkids++] = k;
}

static void xadd_text(xnode *p, char *t) {
    if (p->ntexts == p->captexts) p->texts = (char **)xgrow(p->texts, &p->captexts, sizeof(char *));
    p->texts[p->ntexts++] = t;
}

static void xfree(xnode *x) {
    if (!x) return;
    for (unsigned i = 0; i < x->nkids; ++i) xfree(x->kids[i]);
    for (unsigned i = 0; i < x->ntexts; ++i) free(x->texts[i]);
    free(x->kids);
    free(x->texts);
    free(x->tag);
    free(x);
}

static int starts(const xscan *sc, const char *lit) {
    size_t k = strlen(lit);
    return sc->i + k <= sc->n && memcmp(sc->s + sc->i, lit, k) == 0;
}

/* skip to just past `lit`; 0 when it never comes */
static int skip_past(xscan *sc, const char *lit) {
    size_t k = strlen(lit);
    while (sc->i + k <= sc->n) {
        if (memcmp(sc->s + sc->i, lit, k) == 0) {
            sc->i += k;
            return 1;
        }
        sc->i++;
    }
    sc->i = sc->n;
    return 0;
}

/* append the UTF-8 encoding of code point c */
static size_t put_utf8(char *o, unsigned long c) {
    if (c < 0x80) { o[0] = (char)c; return 1; }
    if (c < 0x800) { o[0] = (char)(0xc0 | (c >> 6)); o[1] = (char)(0x80 | (c & 0x3f)); return 2; }
    if (c < 0x10000) {
        o[0] = (char)(0xe0 | (c >> 12)); o[1] = (char)(0x80 | ((c >> 6) & 0x3f)); o[2] = (char)(0x80 | (c & 0x3f));
        return 3;
    }
    o[0] = (char)(0xf0 | (c >> 18)); o[1] = (char)(0x80 | ((c >> 12) & 0x3f));
    o[2] = (char)(0x80 | ((c >> 6) & 0x3f)); o[3] = (char)(0x80 | (c & 0x3f));
    return 4;
}

/* character data [a, b) with references replaced; `raw` for CDATA */
static char *xtext(const char *a, const char *b, int raw) {
    char *out = (char *)malloc((size_t)(b - a) + 1), *o = out;
    if (!out) abort();
    while (a < b) {
        if (!raw && *a == '&') {
            const char *semi = memchr(a, ';', (size_t)(b - a));
            if (semi) {
                size_t k = (size_t)(semi - a - 1);
                const char *name = a + 1;
                if (k == 2 && !memcmp(name, "lt", 2)) { *o++ = '<'; a = semi + 1; continue; }
                if (k == 2 && !memcmp(name, "gt", 2)) { *o++ = '>'; a = semi + 1; continue; }
                if (k == 3 && !memcmp(name, "amp", 3)) { *o++ = '&'; a = semi + 1; continue; }
                if (k == 4 && !memcmp(name, "quot", 4)) { *o++ = '"'; a = semi + 1; continue; }
                if (k == 4 && !memcmp(name, "apos", 4)) { *o++ = '\''; a = semi + 1; continue; }
                if (k >= 2 && name[0] == '#') {
                    unsigned long c = name[1] == 'x' ? strtoul(name + 2, NULL, 16) : strtoul(name + 1, NULL, 10);
                    o += put_utf8(o, c);   /* at most 4 bytes for the >= 4 bytes read */
                    a = semi + 1;
                    continue;
                }
            }
        }
        *o++ = *a++;
    }
    *o = '\0';
    return out;
}

static int is_name_char(char c) {
    return !(c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '>' || c == '/' || c == '\0');
}

/* the children of `parent` up to its end tag (or the end of input) */
static void xparse_content(xscan *sc, xnode *parent) {
    while (sc->i < sc->n && !sc->bad) {
        if (sc->s[sc->i] != '<') {
            size_t a = sc->i;
            while (sc->i < sc->n && sc->s[sc->i] != '<') sc->i++;
            xadd_text(parent, xtext(sc->s + a, sc->s + sc->i, 0));
            continue;
        }
        if (starts(sc, "<!--")) {
            if (!skip_past(sc, "-->")) sc->bad = 1;
            continue;
        }
        if (starts(sc, "<![CDATA[")) {
            size_t a = sc->i + 9;
            if (!skip_past(sc, "]]>")) { sc->bad = 1; return; }
            xadd_text(parent, xtext(sc->s + a, sc->s + sc->i - 3, 1));
            continue;
        }
        if (starts(sc, "<?")) {
            if (!skip_past(sc, "?>")) sc->bad = 1;
            continue;
        }
        if (starts(sc, "<!")) {   /* DOCTYPE, with an optional [internal subset] */
            int depth = 0;
            while (sc->i < sc->n) {
                char c = sc->s[sc->i++];
                if (c == '[') depth++;
                else if (c == ']') depth--;
                else if (c == '>' && depth <= 0) break;
            }
            continue;
        }
        if (starts(sc, "</")) {   /* the parent's end tag */
            if (!skip_past(sc, ">")) sc->bad = 1;
            return;
        }
        /* a start tag */
        sc->i++;
        size_t a = sc->i;
        while (sc->i < sc->n && is_name_char(sc->s[sc->i])) sc->i++;
        xnode *k = (xnode *)calloc(1, sizeof(xnode));
        if (!k) abort();
        k->tag = xtext(sc->s + a, sc->s + sc->i, 1);
        xadd_kid(parent, k);
        /* attributes: skipped, quoted values may hold '>' */
        int empty = 0;
        while (sc->i < sc->n) {
            char c = sc->s[sc->i];
            if (c == '"' || c == '\'') {
                sc->i++;
                while (sc->i < sc->n && sc->s[sc->i] != c) sc->i++;
                sc->i++;
                continue;
            }
            if (c == '/' && sc->i + 1 < sc->n && sc->s[sc->i + 1] == '>') {
                empty = 1;
                sc->i += 2;
                break;
            }
            sc->i++;
            if (c == '>') break;
        }
        if (!empty) xparse_content(sc, k);
    }
}

static int tag_is(const xnode *x, const char *t) { return strcmp(x->tag, t) == 0; }

/* every descendant element named `t` (XPath .//t), document order */
static void xfind(const xnode *x, const char *t, const xnode ***out, unsigned *n, unsigned *cap) {
    for (unsigned i = 0; i < x->nkids; ++i) {
        if (tag_is(x->kids[i], t)) {
            if (*n == *cap) *out = (const xnode **)xgrow((void *)*out, cap, sizeof(xnode *));
            (*out)[(*n)++] = x->kids[i];
        }
        xfind(x->kids[i], t, out, n, cap);
    }
}

typedef struct {
    const xnode **v;
    unsigned n, cap;
} xlist;

static xlist xall(const xnode *x, const char *t) {
    xlist l = {NULL, 0, 0};
    xfind(x, t, &l.v, &l.n, &l.cap);
    return l;
}

/* the text nodes of every descendant `t` (XPath .//t/text()), in order */
static unsigned xtexts(const xnode *x, const char *t, const char ***out) {
    xlist l = xall(x, t);
    unsigned n = 0, cap = 0;
    *out = NULL;
    for (unsigned i = 0; i < l.n; ++i)
        for (unsigned j = 0; j < l.v[i]->ntexts; ++j) {
            if (n == cap) *out = (const char **)xgrow((void *)*out, &cap, sizeof(char *));
            (*out)[n++] = l.v[i]->texts[j];
        }
    free((void *)l.v);
    return n;
}

/* the NETWORK children named t (XPath //NETWORK/t) */
static xlist network_children(const xnode *root, const char *t) {
    xlist nets = xall(root, "NETWORK"), out = {NULL, 0, 0};
    for (unsigned i = 0; i < nets.n; ++i)
        for (unsigned j = 0; j < nets.v[i]->nkids; ++j)
            if (tag_is(nets.v[i]->kids[j], t)) {
                if (out.n == out.cap) out.v = (const xnode **)xgrow((void *)out.v, &out.cap, sizeof(xnode *));
                out.v[out.n++] = nets.v[i]->kids[j];
            }
    free((void *)nets.v);
    return out;
}

/* the numbers of the TABLE's last text node (count_probabilities /
 * build_probabilities, xml-expression.c:216-276): whitespace-separated
 * tokens, each read with sscanf "%f"; NULL-safe count when out is NULL */
static unsigned table_values(const xnode *defn, float *out, unsigned cap) {
    const char **t = NULL;
    unsigned nt = xtexts(defn, "TABLE", &t);
    assert(nt > 0);
    char *copy = strdup(t[nt - 1]);
    free((void *)t);
    if (!copy) abort();
    unsigned n = 0;
    char *save = NULL;
    for (char *tok = strtok_r(copy, " \t\n\r", &save); tok; tok = strtok_r(NULL, " \t\n\r", &save)) {
        if (out && n < cap) sscanf(tok, "%f", &out[n]);
        n++;
    }
    free(copy);
    return (out && n > cap) ? cap : n;
}

static void name_of(const xnode *x, const char *t, char *buf) {
    const char **txt = NULL;
    unsigned nt = xtexts(x, t, &txt);
    assert(nt == 1);
    strncpy(buf, txt[0], CHAR_BUFFER_SIZE);
    free((void *)txt);
}

static void add_variable(Graph_t graph, const xnode *var) {
    const char **out = NULL;
    unsigned n = xtexts(var, "OUTCOME", &out);
    const unsigned v = graph->current_num_vertices;
    for (unsigned i = 0; i < n; ++i) {
        char *dst = &graph->variable_names[(size_t)v * MAX_STATES * CHAR_BUFFER_SIZE + (size_t)i * CHAR_BUFFER_SIZE];
        strncpy(dst, out[i], CHAR_BUFFER_SIZE);
    }
    free((void *)out);
    char name[CHAR_BUFFER_SIZE];
    name_of(var, "NAME", name);
    graph_add_node(graph, n, name);
}

static void add_prior(Graph_t graph, const xnode *defn) {
    float probs[MAX_STATES];
    for (unsigned i = 0; i < MAX_STATES; ++i) probs[i] = 0.0f;
    const unsigned n = table_values(defn, NULL, 0);
    assert(n < MAX_STATES);
    table_values(defn, probs, n);
    char name[CHAR_BUFFER_SIZE];
    name_of(defn, "FOR", name);
    graph_set_node_state(graph, find_node_by_name(name, graph), n, probs);
}

static void add_edges(Graph_t graph, const xnode *defn, const char **givens, unsigned ng) {
    const unsigned n = table_values(defn, NULL, 0);
    float *total = (float *)malloc(sizeof(float) * (n ? n : 1));
    if (!total) abort();
    table_values(defn, total, n);
    char name[CHAR_BUFFER_SIZE];
    name_of(defn, "FOR", name);
    const unsigned dest = find_node_by_name(name, graph);
    const unsigned ys = graph->node_num_vars[dest];
    const unsigned slice = n / ys;
    unsigned offset = 1;
    float sub[MAX_STATES * MAX_STATES], tr[MAX_STATES * MAX_STATES];
    for (int gi = (int)ng - 1; gi >= 0; --gi) {
        char sname[CHAR_BUFFER_SIZE];
        strncpy(sname, givens[gi], CHAR_BUFFER_SIZE);
        const unsigned src = find_node_by_name(sname, graph);
        const unsigned xs = graph->node_num_vars[src];
        memset(sub, 0, sizeof sub);
        memset(tr, 0, sizeof tr);
        /* the parent's marginal of the CPT, as the reference's strided loop
         * sums it (xml-expression.c:381-395), in the same float order */
        for (unsigned k = 0; k < ys; ++k)
            for (unsigned j = 0; j < xs; ++j) {
                unsigned diff = 0, index = j * offset + diff;
                while (index <= slice) {
                    index = j * offset + diff;
                    const unsigned next = (j + 1) * offset + diff;
                    while (index < next) {
                        const unsigned pos = index + k * slice;
                        sub[j * MAX_STATES + k] += pos < n ? total[pos] : 0.0f;
                        index++;
                    }
                    index += xs * offset;
                    diff += xs * offset;
                }
            }
        for (unsigned j = 0; j < xs; ++j)
            for (unsigned k = 0; k < ys; ++k) tr[k * MAX_STATES + j] = sub[j * MAX_STATES + k];
        graph_add_edge(graph, src, dest, xs, ys, sub);
        if (graph->observed_nodes[src] != 1) graph_add_edge(graph, dest, src, ys, xs, tr);
        offset *= xs;
    }
    free(total);
}

Graph_t parse_xml_file(const char *file_name) {
    FILE *f = fopen(file_name, "rb");
    if (!f) {
        fprintf(stderr, "parse_xml_file: cannot open %s\n", file_name);
        assert(f);
        return NULL;
    }
    fseek(f, 0, SEEK_END);
    long len = ftell(f);
    fseek(f, 0, SEEK_SET);
    char *buf = (char *)malloc((size_t)(len > 0 ? len : 0) + 1);
    if (!buf) abort();
    size_t got = fread(buf, 1, (size_t)(len > 0 ? len : 0), f);
    fclose(f);
    buf[got] = '\0';
    xscan sc = {buf, got, 0, 0};
    xnode *root = (xnode *)calloc(1, sizeof(xnode));
    if (!root) abort();
    root->tag = strdup("");
    xparse_content(&sc, root);
    free(buf);
    assert(!sc.bad);

    xlist vars = network_children(root, "VARIABLE"), defs = network_children(root, "DEFINITION");
    unsigned num_edges = 0;
    for (unsigned i = 0; i < defs.n; ++i)
        for (unsigned j = 0; j < defs.v[i]->nkids; ++j) num_edges += tag_is(defs.v[i]->kids[j], "GIVEN");
    Graph_t graph = create_graph(vars.n, num_edges * 2);
    for (unsigned i = 0; i < vars.n; ++i) add_variable(graph, vars.v[i]);
    for (unsigned i = 0; i < defs.n; ++i) {
        const char **g = NULL;
        if (xtexts(defs.v[i], "GIVEN", &g) == 0) add_prior(graph, defs.v[i]);
        free((void *)g);
    }
    for (unsigned i = 0; i < defs.n; ++i) {
        const char **g = NULL;
        const unsigned ng = xtexts(defs.v[i], "GIVEN", &g);
        if (ng) add_edges(graph, defs.v[i], g, ng);
        free((void *)g);
    }
    free((void *)vars.v);
    free((void *)defs.v);
    xfree(root);
    return graph;
}
