# Prints one top-level C function from a source file: from the line that starts
# with the string in `fn` to the first closing brace in column 0 after it.
index($0, fn) == 1 { on = 1 }
on { print }
on && /^}/ { exit }
