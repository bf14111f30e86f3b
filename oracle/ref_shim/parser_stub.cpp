// The reference reads its input file through a bison/flex parser
// (parser/Parser.y, parser/Lexer.l) that is not generated here: the oracle
// driver fills IoData directly, so the parser entry points are never reached.
#include <cstdio>
#include <cstdlib>
FILE* yyCmdfin = nullptr;
int yyCmdfparse() {
  fprintf(stderr, "oracle: the input-file parser is not built; IoData is filled by the driver\n");
  abort();
}
