"""Extracts the literal golden vectors of the reference's tests.

Reads the reference test sources as text (ast), so it needs no TensorFlow:

  python tests/golden/make_golden.py /path/to/swirl_c > tests/golden/reference_vectors.json

Extracted: the `expected` lists of gradient_test.py
(test_forward_1_provides_correct_1st_order_derivative and
test_central_2_provides_correct_1st_order_derivative).
"""

import ast
import json
import os
import sys


def _expected_list(fn: ast.FunctionDef):
  for node in ast.walk(fn):
    if (isinstance(node, ast.Assign) and len(node.targets) == 1 and
        isinstance(node.targets[0], ast.Name) and
        node.targets[0].id == 'expected' and isinstance(node.value, ast.List)):
      return [ast.literal_eval(e) for e in node.value.elts]
  raise ValueError(f'no literal expected list in {fn.name}')


def main(root: str) -> dict:
  path = os.path.join(root, 'numerics', 'gradient_test.py')
  with open(path) as f:
    tree = ast.parse(f.read())
  out = {'source': 'numerics/gradient_test.py'}
  for node in ast.walk(tree):
    if isinstance(node, ast.FunctionDef):
      if node.name == 'test_forward_1_provides_correct_1st_order_derivative':
        out['gradient_forward_1'] = _expected_list(node)
      elif node.name == 'test_central_2_provides_correct_1st_order_derivative':
        out['gradient_central_2'] = _expected_list(node)
  return out


if __name__ == '__main__':
  print(json.dumps(main(sys.argv[1]), indent=1))
