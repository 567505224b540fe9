"""Writes tests/golden/join_known_answers.json.

The known answers are restated from the reference's own join tests. They were derived by hand
from the SQL semantics those tests assert (DuckDB itself cannot run in this environment):

* test/cpp/integration/test_gpu_execution_join_nulls.cpp:37-43 — the fixture
  l(id, k) = (1,10),(2,20),(3,NULL),(4,30),(5,10); r(id, k) = (1,10),(2,20),(3,20),(4,NULL),(5,40);
  cases :50-104 (INNER, LEFT, RIGHT, FULL, SEMI/ANTI, MARK).
* test/cpp/operator/test_physical_mark_join.cpp:245-530 — operator-level MARK known answers.

Run: python tests/golden/make_golden.py
"""
import json
from pathlib import Path

N = None  # SQL NULL

nulls_fixture = {
    "source": "test/cpp/integration/test_gpu_execution_join_nulls.cpp:37-43",
    "l": {"id": [1, 2, 3, 4, 5], "k": [10, 20, N, 30, 10]},
    "r": {"id": [1, 2, 3, 4, 5], "k": [10, 20, 20, N, 40]},
    # SELECT l.id, r.id FROM l JOIN r ON l.k = r.k   (:50-58)
    "inner": [[1, 1], [2, 2], [2, 3], [5, 1]],
    # ... WHERE l.k IS NULL  -> no rows (:57)
    "inner_where_lk_null": [],
    # LEFT JOIN (:60-65)
    "left": [[1, 1], [2, 2], [2, 3], [3, N], [4, N], [5, 1]],
    # RIGHT JOIN (:67-72)
    "right": [[1, 1], [2, 2], [2, 3], [5, 1], [N, 4], [N, 5]],
    # FULL OUTER JOIN (:74-79)
    "full": [[1, 1], [2, 2], [2, 3], [3, N], [4, N], [5, 1], [N, 4], [N, 5]],
    # EXISTS / NOT EXISTS (:81-89)
    "semi": [1, 2, 5],
    "anti": [3, 4],
    # l.k IN (SELECT k FROM r): build side has a NULL (:91-104)
    "mark_with_null_build": [[1, True], [2, True], [3, N], [4, N], [5, True]],
    # l.k IN (SELECT k FROM r WHERE k IS NOT NULL)
    "mark_null_free_build": [[1, True], [2, True], [3, N], [4, False], [5, True]],
    # IS NOT DISTINCT FROM on the same data: NULL matches NULL
    # (test/cpp/integration/test_gpu_execution_null_safe_join.cpp pins the null-safe rule)
    "inner_null_safe": [[1, 1], [2, 2], [2, 3], [3, 4], [5, 1]],
}

mark_cases = [
    {"name": "partial match", "source": "test_physical_mark_join.cpp:245-274",
     "left": [10, 20, 30, 40, 50], "right": [20, 40], "mark": [False, True, False, True, False]},
    {"name": "all rows match", "source": "test_physical_mark_join.cpp:276-303",
     "left": [10, 20, 30], "right": [10, 20, 30], "mark": [True, True, True]},
    {"name": "no rows match", "source": "test_physical_mark_join.cpp:305-332",
     "left": [10, 20, 30], "right": [40, 50, 60], "mark": [False, False, False]},
    {"name": "empty right side", "source": "test_physical_mark_join.cpp:334-361",
     "left": [10, 20, 30], "right": [], "mark": [False, False, False]},
    {"name": "duplicate keys on right side", "source": "test_physical_mark_join.cpp:363-391",
     "left": [10, 20, 30], "right": [20, 20, 20], "mark": [False, True, False]},
    {"name": "build-on-left path", "source": "test_physical_mark_join.cpp:393-427",
     "left": [10, 20, 30, 40], "right": [20, 40, 11, 12, 13, 14, 15, 16], "mark": [False, True, False, True]},
    {"name": "right side has NULL key", "source": "test_physical_mark_join.cpp:429-457",
     "left": [1, 2, 3], "right": [2, N], "mark": [N, True, N]},
    {"name": "probe side has NULL key", "source": "test_physical_mark_join.cpp:459-491",
     "left": [1, N, 2], "right": [2], "mark": [False, N, True]},
    {"name": "right NULL key on build-on-left path", "source": "test_physical_mark_join.cpp:493-526",
     "left": [10, 20, 30, 40], "right": [20, 40, N, 11, 12, 13, 14], "mark": [N, True, N, True]},
]

out = {"nulls_fixture": nulls_fixture, "mark_cases": mark_cases}
path = Path(__file__).resolve().parent / "join_known_answers.json"
path.write_text(json.dumps(out, indent=1) + "\n")
print(path)
